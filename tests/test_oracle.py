"""Pins the CPU oracle to the reference's own tests (CPU only).

- the three golden final fields of test/test2D_xPU.jl:108-195, with the
  reference's comparison (isapprox, rtol sqrt(eps));
- the update_ψ! known-answer tests of test/test2D.jl:13-43 and
  test/test3D.jl:13-71;
- the analytic Green's-function tests of test/test2D_xPU.jl:12-106 and
  test/test3D_xPU.jl:12-108 (trace vs the homogeneous-medium solution,
  integrated absolute error <= 1% of the peak times lt).
"""
import math

import numpy as np
import pytest

import cases


def _run(oracle, case):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    s = oracle.setup(lengths, lt, vel, sp, t0s, f0, rp, **kw)
    return s, oracle.forward(s)


@pytest.mark.parametrize("name,case", [
    ("acoustic2D_center_halo20", lambda: cases.ref_center(False)),
    ("acoustic2D_center_freetop_halo20", lambda: cases.ref_center(True)),
    ("acoustic2D_gradient_freetop_halo20", cases.ref_gradient),
])
def test_oracle_matches_reference_golden(oracle, name, case):
    s, (pend, _) = _run(oracle, case())
    ref = cases.golden(name)
    assert pend.shape == ref.shape
    assert cases.isapprox(pend, ref), cases.rel_l2(pend, ref)
    # the oracle restates the arithmetic, so it is far inside the tolerance
    assert cases.rel_l2(pend, ref) < 1e-10


def test_gradient_case_sources_sit_on_dirichlet_row(oracle):
    s = oracle.setup(*cases.ref_gradient()[:7], **cases.ref_gradient()[7])
    assert np.all(s["possrcs"][:, 1] == 1)


def test_update_psi_known_answer_2d(oracle):
    # test/test2D.jl:13-43
    nx = ny = 101
    halo = 20
    pcur = np.ones((nx, ny), order="F")
    pcur[[0, -1], :] = 0.0
    pcur[:, [0, -1]] = 0.0
    psi = [np.ones((halo + 1, ny), order="F"), np.ones((halo + 1, ny), order="F"),
           np.ones((nx, halo + 1), order="F"), np.ones((nx, halo + 1), order="F")]
    half, two = 0.5 * np.ones(halo + 1), 2.0 * np.ones(halo + 1)
    oracle.update_psi(pcur, halo, [0.1, 0.1], psi, [half, two, half, two] * 2)
    pxl, pxr, pyl, pyr = psi
    assert np.array_equal(pxl[0, :], [0.5] + [0.55] * (ny - 2) + [0.5])
    assert np.array_equal(pxl[1:, :], 0.5 * np.ones((halo, ny)))
    assert np.array_equal(pxr[:-1, :], 2.0 * np.ones((halo, ny)))
    assert np.array_equal(pxr[-1, :], [2.0] + [1.8] * (ny - 2) + [2.0])
    assert np.array_equal(pyl[:, 0], [0.5] + [0.55] * (nx - 2) + [0.5])
    assert np.array_equal(pyl[:, 1:], 0.5 * np.ones((nx, halo)))
    assert np.array_equal(pyr[:, :-1], 2.0 * np.ones((nx, halo)))
    assert np.array_equal(pyr[:, -1], [2.0] + [1.8] * (nx - 2) + [2.0])


def test_update_psi_known_answer_3d(oracle):
    # test/test3D.jl:13-71
    n = 101
    halo = 20
    pcur = np.ones((n, n, n), order="F")
    pcur[[0, -1], :, :] = 0.0
    pcur[:, [0, -1], :] = 0.0
    pcur[:, :, [0, -1]] = 0.0
    shp = [(halo + 1, n, n), (n, halo + 1, n), (n, n, halo + 1)]
    psi = [np.ones(shp[a // 2], order="F") for a in range(6)]
    half, two = 0.5 * np.ones(halo + 1), 2.0 * np.ones(halo + 1)
    oracle.update_psi(pcur, halo, [0.1, 0.1, 0.1], psi, [half, two, half, two] * 3)
    a1 = 0.55 * np.ones((n, n))
    a1[[0, -1], :] = 0.5
    a1[:, [0, -1]] = 0.5
    a2 = 1.8 * np.ones((n, n))
    a2[[0, -1], :] = 2.0
    a2[:, [0, -1]] = 2.0
    assert np.array_equal(psi[0][0, :, :], a1)
    assert np.array_equal(psi[0][1:, :, :], 0.5 * np.ones((halo, n, n)))
    assert np.array_equal(psi[1][:-1, :, :], 2.0 * np.ones((halo, n, n)))
    assert np.array_equal(psi[1][-1, :, :], a2)
    assert np.array_equal(psi[2][:, 0, :], a1)
    assert np.array_equal(psi[2][:, 1:, :], 0.5 * np.ones((n, halo, n)))
    assert np.array_equal(psi[3][:, :-1, :], 2.0 * np.ones((n, halo, n)))
    assert np.array_equal(psi[3][:, -1, :], a2)
    assert np.array_equal(psi[4][:, :, 0], a1)
    assert np.array_equal(psi[4][:, :, 1:], 0.5 * np.ones((n, n, halo)))
    assert np.array_equal(psi[5][:, :, :-1], 2.0 * np.ones((n, n, halo)))
    assert np.array_equal(psi[5][:, :, -1], a2)


def _trapz(x, y):
    return float(np.sum(0.5 * (y[1:] + y[:-1]) * np.diff(x)))


def analytic_trace_2d(dt, nt, dist, c0, t0, f0):
    """test/test2D_xPU.jl:34-53: 2D Green's function convolved with the source."""
    times = np.arange(nt + 1) * dt
    G = np.zeros(nt + 1)
    m = times - dist / c0 >= 0
    G[m] = 1.0 / (2 * math.pi * c0 ** 2 * np.sqrt(times[m] ** 2 - dist ** 2 / c0 ** 2))
    src = _ricker(times, t0, f0)
    Gc = np.convolve(G, src * dt)[1:nt + 1]
    return times, Gc


def analytic_trace_3d(dt, nt, dist, c0, t0, f0):
    """test/test3D_xPU.jl:35-54: delta Green's function 1/(4 pi c^2 r)."""
    times = np.arange(nt + 1) * dt
    G = np.zeros(nt + 1)
    idx = np.nonzero(times - dist / c0 >= 0)[0]
    if idx.size:
        G[idx[0]] = 1.0 / (4 * math.pi * c0 ** 2 * dist)
    src = _ricker(times, t0, f0)
    Gc = np.convolve(G, src)[1:nt + 1]
    return times, Gc


def _ricker(t, t0, f0):
    x = math.pi * f0 * (t - t0)
    return (1 - 2 * x * x) * np.exp(-x * x)


def analytic_case_2d(halo):
    n, L, c0, f0 = 501, 10.0, 1.0, 1.0
    lt = 10.0 if halo == 0 else 20.0
    return ((L, L), lt, c0 * np.ones((n, n)), [[L / 2, L / 2]], [4 / f0], f0, [[L / 4, L / 2]],
            dict(halo=halo, rcoef=1e-4, freetop=False))


def analytic_case_3d(halo):
    n, L, c0, f0 = 101, 20.0, 1.0, 0.25
    lt = 26.0 if halo == 0 else 50.0
    return ((L, L, L), lt, c0 * np.ones((n, n, n)), [[L / 2, L / 2, L / 2]], [4 / f0], f0,
            [[L / 4, L / 2, L / 2]], dict(halo=halo, rcoef=1e-4, freetop=False))


def check_analytic(trace, s, case, ndim):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    dist = float(np.linalg.norm(np.subtract(sp[0], rp[0])))
    fn = analytic_trace_2d if ndim == 2 else analytic_trace_3d
    times, Gc = fn(s["dt"], s["nt"], dist, 1.0, t0s[0], f0)
    assert len(trace) == len(Gc) == s["nt"]
    err = _trapz(times[1:], np.abs(trace - Gc))
    bound = np.max(np.abs(Gc)) * 0.01 * lt
    assert err <= bound, (err, bound)
    return err / bound


@pytest.mark.parametrize("halo", [0, 20])
def test_oracle_analytic_2d(oracle, halo):
    case = analytic_case_2d(halo)
    s, (_, traces) = _run(oracle, case)
    check_analytic(traces[:, 0], s, case, 2)


@pytest.mark.parametrize("halo", [0, 20])
def test_oracle_analytic_3d(oracle, halo):
    case = analytic_case_3d(halo)
    s, (_, traces) = _run(oracle, case)
    check_analytic(traces[:, 0], s, case, 3)


# ---- 1D (src/shared/acoustic_1D.jl, test/test1D.jl) --------------------------

def analytic_case_1d(halo):
    """test/test1D.jl:7-52 (halo 0, lt = 10) and :54-99 (halo 20, lt = 20):
    1001 nodes on 10 m, c0 = 1, Ricker f0 = 1 Hz, t0 = 4 s, source at lx/2,
    receiver at lx/4."""
    nx, lx = 1001, 10.0
    return ((lx,), 10.0 if halo == 0 else 20.0, np.ones(nx), [[lx / 2]], [4.0], 1.0,
            [[lx / 4]], dict(halo=halo, rcoef=1e-4, freetop=False))


def analytic_trace_1d(dt, nt, dist, c0, t0, f0):
    """test/test1D.jl:30-47: Heaviside Green's function 1/(2 c0) after the
    arrival, convolved with the source times dt."""
    times = np.arange(nt + 1) * dt
    G = np.where(times - dist / c0 >= 0, 1.0 / (2 * c0), 0.0)
    src = _ricker(times, t0, f0)
    Gc = np.convolve(G, src * dt)[1:nt + 1]
    return times, Gc


@pytest.mark.parametrize("halo", [0, 20])
def test_oracle_analytic_1d(oracle, halo):
    lengths, lt, vel, sp, t0s, f0, rp, kw = analytic_case_1d(halo)
    s = oracle.setup(lengths, lt, vel, sp, t0s, f0, rp, **kw)
    assert s["dt"] == 10.0 / 1000 / 1.0 / 2
    _, tr = oracle.forward_1d(s)
    times, Gc = analytic_trace_1d(s["dt"], s["nt"], abs(sp[0][0] - rp[0][0]), 1.0, t0s[0], f0)
    assert len(Gc) == s["nt"] == tr.shape[0]
    err = _trapz(times[1:], np.abs(tr[:, 0] - Gc))
    assert err <= np.max(np.abs(Gc)) * 0.01 * lt, err


def test_oracle_1d_cpml_absorbs(oracle):
    """With the CPML the 1D pulse leaves the line: after both arrivals the
    field is far below its peak (without a band it stays reflected)."""
    lengths, lt, vel, sp, t0s, f0, rp, kw = analytic_case_1d(20)
    s = oracle.setup(lengths, 30.0, vel, sp, t0s, f0, rp, **kw)
    pend, tr = oracle.forward_1d(s)
    s0 = oracle.setup(lengths, 30.0, vel, sp, t0s, f0, rp, **dict(kw, halo=0))
    pend0, _ = oracle.forward_1d(s0)
    assert np.abs(pend).max() < 1e-2 * np.abs(tr).max()
    assert np.abs(pend0).max() > 0.1 * np.abs(tr).max()
