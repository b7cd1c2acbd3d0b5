"""Source/receiver types, the Ricker wavelet and the CPML profile.

Mirrors the user-facing helpers of AcousticWaveCPML.jl's src/utils.jl
(`Sources` :88-121, `Receivers` :126-145, `rickersource1D` :64-66,
`calc_Kab_CPML` :19-57) with the same argument meaning and the same
assertion errors. The CPML profile is computed by the C library (FP64).
"""
import math

import numpy as np

from . import _lib


class Sources:
    """Multi-source configuration of one shot (src/utils.jl:88-121).

    positions: (nsrc, ndim) metres; t0s: activation times [s]; srctfs: one
    callable (t, t0, f0) per source; freqdomain: the dominating frequency f0.
    """

    def __init__(self, positions, t0s, srctfs, freqdomain):
        positions = np.atleast_2d(np.asarray(positions, dtype=np.float64))
        assert positions.shape[0] > 0, "There must be at least one source!"
        assert positions.shape[0] == len(t0s) == len(srctfs), \
            "Number of sources do not match between positions and time-functions!"
        self.n = positions.shape[0]
        self.positions = positions
        self.t0s = [float(t) for t in t0s]
        self.srctfs = list(srctfs)
        self.freqdomain = float(freqdomain)


class Receivers:
    """Receiver configuration (src/utils.jl:126-145); `seismograms` is filled
    by the solvers with one column per receiver and one row per time step."""

    def __init__(self, positions):
        positions = np.atleast_2d(np.asarray(positions, dtype=np.float64))
        assert positions.shape[0] > 0, "There must be at least one receiver!"
        self.n = positions.shape[0]
        self.positions = positions
        self.seismograms = np.zeros((0, 0))


def rickersource1D(t, t0, f0):
    """Ricker wavelet (src/utils.jl:64-66); `t` may be a scalar or an array."""
    x = math.pi * f0 * (np.asarray(t, dtype=np.float64) - t0)
    return (1.0 - 2.0 * (x * x)) * np.exp(-(x * x))


def calc_Kab_CPML(halo, dt, npower, d0, alpha_max_pml, K_max_pml, onwhere):
    """K, a, b CPML coefficients (src/utils.jl:19-57).

    Returns (a_left, a_right, b_K_left, b_K_right); length `halo` for
    onwhere="ongrd", halo+1 for "halfgrd"."""
    if onwhere == "halfgrd":
        n, half = halo + 1, 1
    elif onwhere == "ongrd":
        n, half = halo, 0
    else:
        raise ValueError("Wrong onwhere parameter!")
    out = [np.zeros(n) for _ in range(4)]
    dp = [o.ctypes.data_as(_lib._dp) for o in out]
    _lib.check(_lib.lib().awc_cpml_coeffs(int(halo), float(dt), float(npower), float(d0),
                                          float(alpha_max_pml), float(K_max_pml), half, *dp))
    return tuple(out)
