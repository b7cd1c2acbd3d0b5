"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is an FP64 C++ restatement of AcousticWaveCPML.jl's xPU solver
(oracle/awc_oracle.cpp). This module adds a numpy restatement of the host setup
that solve2D/solve3D perform before their time loop
(src/shared/acoustic_2D_xPU.jl:154-240, src/shared/acoustic_3D_xPU.jl:194-289):
dt and nt from the CFL rule, the ricker source time functions scaled by
dt^2/(dx dy [dz]), and the nearest-node snapping of positions. It is used by
the tests, the smoke check and the CPU-baseline leg of bench.py as the checker;
the product never imports it.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


class Problem(ctypes.Structure):
    """Mirror of `awc_problem` in include/awcpml.h."""

    _fields_ = [
        ("ndim", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("halo", ctypes.c_int32),
        ("freetop", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("nt", ctypes.c_int64),
        ("nsrc", ctypes.c_int64),
        ("nrec", ctypes.c_int64),
    ]


def _has_avx2():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx2 " in line + " "
    except OSError:
        pass
    return False


_LIB = None


def lib():
    """Loads oracle/build/libawc_oracle[_avx2].so (built by `make -C oracle`)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    names = ["libawc_oracle_avx2.so", "libawc_oracle.so"] if _has_avx2() else ["libawc_oracle.so"]
    for n in names:
        path = os.path.join(_HERE, "build", n)
        if os.path.exists(path):
            L = ctypes.CDLL(path)
            break
    else:
        raise RuntimeError("oracle library not built: run `make -C oracle`")
    dp = ctypes.POINTER(ctypes.c_double)
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.oracle_calc_Kab_CPML.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, dp, dp, dp, dp]
    L.oracle_ricker.argtypes = [ctypes.c_double] * 3
    L.oracle_ricker.restype = ctypes.c_double
    L.oracle_problem_coeffs.argtypes = [ctypes.POINTER(Problem), ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, dp]
    L.oracle_update_psi.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.c_int64, ctypes.c_int32, dp, dp,
                                    ctypes.POINTER(dp), ctypes.POINTER(dp)]
    L.oracle_forward.argtypes = [ctypes.POINTER(Problem), dp, dp, i64p, dp, i64p, dp, dp,
                                 ctypes.c_int32, ctypes.c_int64]
    L.oracle_max_threads.restype = ctypes.c_int
    L.oracle_last_loop_seconds.restype = ctypes.c_double
    _LIB = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def calc_Kab_CPML(halo, dt, npower, d0, alpha_max_pml, K_max_pml, onwhere):
    """calc_Kab_CPML (src/utils.jl:19-57) through the C restatement."""
    if onwhere not in ("ongrd", "halfgrd"):
        raise ValueError("Wrong onwhere parameter!")
    n = halo + (1 if onwhere == "halfgrd" else 0)
    out = [np.zeros(n) for _ in range(4)]
    lib().oracle_calc_Kab_CPML(halo, dt, npower, d0, alpha_max_pml, K_max_pml,
                               1 if onwhere == "halfgrd" else 0, *[_dp(o) for o in out])
    return tuple(out)


def ricker(t, t0, f0):
    """rickersource1D (src/utils.jl:64-66), vectorised over t."""
    x = math.pi * f0 * (np.asarray(t, dtype=np.float64) - t0)
    return (1.0 - 2.0 * (x * x)) * np.exp(-(x * x))


def round_ties_up(x):
    """round(Int, x, RoundNearestTiesUp) for finite x."""
    x = np.asarray(x, dtype=np.float64)
    f = np.floor(x)
    return (f + ((x - f) >= 0.5)).astype(np.int64)


def setup(lengths, lt, vel, src_positions, t0s, f0, rec_positions, halo=20, rcoef=1e-4,
          ppw=10.0, freetop=True, dt=None, nt=None, check_ppw=True):
    """Host setup of solve2D/solve3D (acoustic_3D_xPU.jl:194-289).

    `lengths` = (lx, ly[, lz]); `vel` is indexed vel[i, j[, k]] (any memory
    order; it is copied column-major). When `dt`/`nt` are given they replace
    the CFL-derived values (a fixed-dt configuration); otherwise the
    reference's rule is used. Returns a dict with the Problem and the arrays
    awc_forward / oracle_forward take.
    """
    vel = np.asfortranarray(vel, dtype=np.float64)
    ndim = vel.ndim
    assert ndim in (1, 2, 3) and len(lengths) == ndim
    if ndim == 1:
        freetop = False  # acoustic_1D.jl has no free top
    shape = vel.shape
    vel_max = float(vel.max())
    d = [lengths[a] / (shape[a] - 1) for a in range(ndim)]
    if dt is None:
        inv = sum(1.0 / x for x in d)
        dt = math.sqrt(ndim) / (vel_max * inv) / 2.0
    if nt is None:
        nt = int(math.ceil(lt / dt))
    if check_ppw:
        assert math.sqrt(sum(x * x for x in d)) <= vel_max / (ppw * f0), \
            "Not enough points per wavelength!"
    times = np.arange(nt, dtype=np.float64) * dt
    src_positions = np.atleast_2d(np.asarray(src_positions, dtype=np.float64))
    rec_positions = np.atleast_2d(np.asarray(rec_positions, dtype=np.float64))
    nsrc, nrec = src_positions.shape[0], rec_positions.shape[0]
    scale = (dt * dt) / math.prod(d)
    dt2srctf = np.zeros((nt, nsrc), order="F")
    for s in range(nsrc):
        dt2srctf[:, s] = scale * ricker(times, t0s[s], f0)

    def snap(pos):
        out = np.zeros(pos.shape, dtype=np.int64, order="F")
        for a in range(ndim):
            out[:, a] = round_ties_up(pos[:, a] / d[a] + 1.0)
        for a in range(ndim):
            assert np.all((out[:, a] >= 1) & (out[:, a] <= shape[a])), "not inside the model"
        return out

    possrcs, posrecs = snap(src_positions), snap(rec_positions)
    p = Problem(ndim=ndim, precision=2, nx=shape[0], ny=shape[1] if ndim >= 2 else 1,
                nz=shape[2] if ndim == 3 else 1, halo=halo, freetop=1 if freetop else 0,
                dx=d[0], dy=d[1] if ndim >= 2 else 1.0, dz=d[2] if ndim == 3 else 1.0, dt=dt,
                nt=nt, nsrc=nsrc, nrec=nrec)
    coeffs = problem_coeffs(p, rcoef, f0, vel_max)
    return dict(problem=p, vel=vel, coeffs=coeffs, possrcs=np.asfortranarray(possrcs),
                dt2srctf=dt2srctf, posrecs=np.asfortranarray(posrecs), dt=dt, nt=nt,
                d=d, vel_max=vel_max)


def problem_coeffs(p, rcoef, f0, vel_max):
    n = p.ndim * (8 * p.halo + 4)
    coeffs = np.zeros(n)
    if p.ndim == 1:
        # solve1D's CPML block (acoustic_1D.jl:118-125), the x block of 2D
        q = Problem.from_buffer_copy(p)
        q.ndim, q.ny, q.dy, q.freetop = 2, 3, p.dx, 0
        c2 = np.zeros(2 * (8 * p.halo + 4))
        lib().oracle_problem_coeffs(ctypes.byref(q), rcoef, f0, vel_max, _dp(c2))
        coeffs[:] = c2[:n]
        return coeffs
    lib().oracle_problem_coeffs(ctypes.byref(p), rcoef, f0, vel_max, _dp(coeffs))
    return coeffs


def forward(s, nthreads=0, steps=-1):
    """Runs oracle_forward on a setup() dict. Returns (pfinal, traces)."""
    p = s["problem"]
    shape = (p.nx, p.ny) if p.ndim == 2 else (p.nx, p.ny, p.nz)
    traces = np.zeros((p.nt, p.nrec), order="F")
    pfinal = np.zeros(shape, order="F")
    vel = np.asfortranarray(s["vel"], dtype=np.float64)
    rc = lib().oracle_forward(ctypes.byref(p), _dp(vel), _dp(s["coeffs"]), _i64p(s["possrcs"]),
                              _dp(s["dt2srctf"]), _i64p(s["posrecs"]), _dp(traces), _dp(pfinal),
                              int(nthreads), int(steps))
    assert rc == 0
    return pfinal, traces


def update_psi(pcur, halo, inv_d, psi, coef):
    """update_ψ! of the serial solvers on caller arrays (in place).

    psi = [ψx_l, ψx_r, ψy_l, ψy_r(, ψz_l, ψz_r)] Fortran-ordered float64 arrays;
    coef = [a_xhl, a_xhr, bK_xhl, bK_xhr, a_yhl, ...] (4 per axis)."""
    pcur = np.asfortranarray(pcur, dtype=np.float64)
    ndim = pcur.ndim
    shape = pcur.shape + ((1,) if ndim == 2 else ())
    for a in psi:
        assert a.flags.f_contiguous and a.dtype == np.float64
    coef = [np.ascontiguousarray(c, dtype=np.float64) for c in coef]
    d = np.asarray(list(inv_d) + [1.0] * (3 - len(inv_d)), dtype=np.float64)
    PsiArr = ctypes.POINTER(ctypes.c_double) * 6
    CoefArr = ctypes.POINTER(ctypes.c_double) * 12
    pa = PsiArr(*([_dp(a) for a in psi] + [None] * (6 - len(psi))))
    ca = CoefArr(*([_dp(c) for c in coef] + [None] * (12 - len(coef))))
    lib().oracle_update_psi(ndim, shape[0], shape[1], shape[2], halo, _dp(pcur), _dp(d), pa, ca)


def max_threads():
    return lib().oracle_max_threads()


def last_loop_seconds():
    return lib().oracle_last_loop_seconds()


def forward_1d(s):
    """FP64 numpy restatement of the reference's 1D solver on a setup() dict
    of a 1D problem (src/shared/acoustic_1D.jl): per step update_ψ! (:7-19,
    both CPML ends, ψ on the half grid), update_p! (:21-48, ξ and the damping
    term in the bands, i <= halo+1 and i >= nx-halo in 1-based indices),
    inject_sources! (:50-56), record_receivers! (:58-64) and the
    (pold, pcur, pnew) <- (pcur, pnew, pold) rotation of forward! (:66-88).
    Returns (pfinal, traces)."""
    p = s["problem"]
    nx, h, nt = p.nx, p.halo, p.nt
    dx = p.dx
    _dx, _dx2 = 1.0 / dx, 1.0 / (dx * dx)
    c = s["coeffs"]
    a_l, a_r, bK_l, bK_r = c[0:h], c[h:2 * h], c[2 * h:3 * h], c[3 * h:4 * h]
    hb = c[4 * h:]
    a_hl, a_hr = hb[0:h + 1], hb[h + 1:2 * (h + 1)]
    bK_hl, bK_hr = hb[2 * (h + 1):3 * (h + 1)], hb[3 * (h + 1):4 * (h + 1)]
    fact = (p.dt * p.dt) * np.asarray(s["vel"], dtype=np.float64) ** 2
    pold, pcur, pnew = np.zeros(nx), np.zeros(nx), np.zeros(nx)
    psi_l, psi_r = np.zeros(h + 1), np.zeros(h + 1)
    xi_l, xi_r = np.zeros(h), np.zeros(h)
    src = np.asarray(s["possrcs"])[:, 0] - 1
    rec = np.asarray(s["posrecs"])[:, 0] - 1
    stf = s["dt2srctf"]
    traces = np.zeros((nt, p.nrec), order="F")
    i_in = np.arange(1, nx - 1)  # 0-based interior nodes
    for it in range(nt):
        # update_ψ!: entries i = 1..halo+1 (1-based), right side shifted
        if h > 0:
            q = np.arange(h + 1)
            ii = q + nx - h - 2
            psi_l = bK_hl * psi_l + a_hl * (pcur[q + 1] - pcur[q]) * _dx
            psi_r = bK_hr * psi_r + a_hr * (pcur[ii + 1] - pcur[ii]) * _dx
        # update_p!
        d2p = (pcur[i_in + 1] - 2.0 * pcur[i_in] + pcur[i_in - 1]) * _dx2  # d2p[i0 - 1]
        damp = np.zeros(nx - 2)
        if h > 0:
            # left band: 1-based i = 2 .. halo+1 (ψ entries i, i-1; ξ entry i-1)
            il = np.arange(2, min(h + 1, nx - 1) + 1)
            dpsi = (psi_l[il - 1] - psi_l[il - 2]) * _dx
            xi_l[il - 2] = bK_l[il - 2] * xi_l[il - 2] + a_l[il - 2] * (d2p[il - 2] + dpsi)
            damp[il - 2] = fact[il - 1] * (dpsi + xi_l[il - 2])
            # right band: nx-halo <= i <= nx-1, not already in the left band
            ir = np.arange(max(nx - h, h + 2), nx)
            ii = ir - (nx - h) + 2
            dpsi = (psi_r[ii - 1] - psi_r[ii - 2]) * _dx
            xi_r[ii - 2] = bK_r[ii - 2] * xi_r[ii - 2] + a_r[ii - 2] * (d2p[ir - 2] + dpsi)
            damp[ir - 2] = fact[ir - 1] * (dpsi + xi_r[ii - 2])
        pnew[i_in] = 2.0 * pcur[i_in] - pold[i_in] + fact[i_in] * d2p + damp
        for k, node in enumerate(src):
            pnew[node] += stf[it, k]
        for r, node in enumerate(rec):
            traces[it, r] = pnew[node]
        pold, pcur, pnew = pcur, pnew, pold
    return pcur.copy(), traces
