"""GPU forward solve through the C ABI vs the oracle and the reference's
golden fields. Tolerances (relative L2): FP64 build <= 1e-10 against the
FP64 oracle on traces and the final field; FP32 build <= 1e-4 on traces.
The golden fields also use the reference's own criterion (isapprox)."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4


def run_both(pkg, oracle, ctx, case, precision):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    kw = dict(kw)
    check_ppw = kw.pop("check_ppw", True)
    if not check_ppw:
        kw_p = dict(kw, ppw=1e-9)
    else:
        kw_p = kw
    s = pkg.prepare(lengths, lt, vel, srcs, recs, precision=precision, **kw_p)
    p = s["problem"]
    traces = np.zeros((p.nt, p.nrec), order="F")
    pend = np.zeros(s["vel"].shape, order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], traces, pend)
    so = oracle.setup(lengths, lt, vel, sp, t0s, f0, rp, check_ppw=check_ppw, **kw)
    pend_o, traces_o = oracle.forward(so)
    return s, (pend, traces), (pend_o, traces_o)


GOLDEN = [
    ("acoustic2D_center_halo20", lambda: cases.ref_center(False)),
    ("acoustic2D_center_freetop_halo20", lambda: cases.ref_center(True)),
    ("acoustic2D_gradient_freetop_halo20", cases.ref_gradient),
]


@pytest.mark.parametrize("name,case", GOLDEN)
def test_golden_2d_f64(pkg, oracle, ctx, name, case):
    s, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, case(), "f64")
    ref = cases.golden(name)
    assert cases.isapprox(pend, ref), cases.rel_l2(pend, ref)
    assert cases.rel_l2(pend, pend_o) <= TOL64
    assert cases.rel_l2(traces, traces_o) <= TOL64


@pytest.mark.parametrize("name,case", GOLDEN)
def test_golden_2d_f32(pkg, oracle, ctx, name, case):
    s, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, case(), "f32")
    e = cases.rel_l2(traces, traces_o)
    print(f"{name} f32 traces rel-L2 {e:.3e} field {cases.rel_l2(pend, pend_o):.3e}")
    assert e <= TOL32


def _w2case(w):
    return (w["lengths"], w["lt"], w["vel"], w["src_pos"], w["t0s"], w["f0"], w["rec_pos"],
            w["kwargs"])


@pytest.mark.parametrize("precision,tol", [("f64", TOL64), ("f32", TOL32)])
def test_config1_2d(pkg, oracle, ctx, precision, tol):
    from acousticwavecpml_b200 import workloads as W
    s, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, _w2case(W.config1()),
                                                     precision)
    e = cases.rel_l2(traces, traces_o)
    print(f"config1 {precision}: traces rel-L2 {e:.3e}, field {cases.rel_l2(pend, pend_o):.3e}")
    assert e <= tol
    if precision == "f64":
        assert cases.rel_l2(pend, pend_o) <= tol


def small3d(n=(40, 34, 28), halo=6, freetop=True, srcs=None, recs=None, lt=0.2, seed=0):
    nx, ny, nz = n
    d = 10.0
    rng = np.random.default_rng(seed)
    vel = 2000.0 + 15.0 * np.arange(ny)[None, :, None] + 50.0 * rng.random((nx, ny, nz))
    L = ((nx - 1) * d, (ny - 1) * d, (nz - 1) * d)
    f0 = 12.0
    if srcs is None:
        srcs = [[(nx // 2) * d, 8 * d, (nz // 2) * d]]
    if recs is None:
        recs = [[(i - 1) * d, 3 * d, (k - 1) * d] for i in (3, nx // 2, nx - 3) for k in (4, nz - 4)]
        recs += [[(nx // 3) * d, (ny - 5) * d, (nz // 3) * d]]
    # the wavelet peaks at t0 = 0.05 s, inside every case's lt, so the fields
    # are far above FP32's range floor from the first steps on
    return (L, lt, vel, srcs, [0.05] * len(srcs), f0, recs,
            dict(halo=halo, rcoef=1e-4, freetop=freetop, check_ppw=False))


CASES3D = {
    "freetop": lambda: small3d(),
    "cpml_all_sides": lambda: small3d(freetop=False),
    "halo0": lambda: small3d(halo=0),
    "halo1": lambda: small3d(halo=1, freetop=False),
    # sources and receivers on Dirichlet rows (energy enters only through
    # the rim accumulation, as in the reference's gradient test)
    "rim_sources": lambda: small3d(srcs=[[100.0, 0.0, 100.0], [0.0, 50.0, 60.0],
                                         [390.0, 330.0, 270.0]],
                                   recs=[[100.0, 0.0, 100.0], [200.0, 30.0, 100.0]]),
    # several sources on one node are summed
    "duplicate_sources": lambda: small3d(srcs=[[200.0, 80.0, 140.0]] * 3 + [[120.0, 90.0, 90.0]]),
    # left and right bands overlap (n < 2 halo + 2)
    "overlapping_bands": lambda: small3d(n=(12, 11, 13), halo=5, freetop=False,
                                         srcs=[[50.0, 50.0, 60.0]], recs=[[20.0, 20.0, 30.0]],
                                         lt=0.1),
    "odd_sizes": lambda: small3d(n=(37, 45, 19), halo=4, freetop=True),
    "thin_z": lambda: small3d(n=(70, 40, 5), halo=1, freetop=False,
                              srcs=[[300.0, 200.0, 20.0]], recs=[[100.0, 100.0, 20.0]]),
    # a core box with all three band launches around it (x band tiles, y band
    # rows, z band planes), sources and receivers in each part
    "core_and_bands": lambda: small3d(
        n=(100, 90, 80), halo=20, freetop=False, lt=0.12,
        srcs=[[490.0, 400.0, 390.0], [100.0, 450.0, 300.0], [500.0, 820.0, 100.0]],
        recs=[[(i - 1) * 10.0, (j - 1) * 10.0, (k - 1) * 10.0]
              for i, j, k in ((5, 5, 5), (30, 40, 40), (60, 85, 40), (97, 45, 78), (50, 45, 10),
                              (33, 40, 40), (64, 70, 21), (65, 70, 60), (2, 2, 2))]),
    # a halo wider than one 32-node x tile, free top
    "wide_halo_freetop": lambda: small3d(n=(133, 70, 90), halo=34, freetop=True, lt=0.1,
                                         srcs=[[660.0, 300.0, 450.0], [100.0, 30.0, 50.0]]),
}


@pytest.mark.parametrize("name", sorted(CASES3D))
@pytest.mark.parametrize("precision,tol", [("f64", TOL64), ("f32", TOL32)])
def test_3d_cases(pkg, oracle, ctx, name, precision, tol):
    s, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, CASES3D[name](), precision)
    e_t = cases.rel_l2(traces, traces_o)
    e_p = cases.rel_l2(pend, pend_o)
    print(f"{name} {precision}: traces {e_t:.3e} field {e_p:.3e}")
    assert np.all(np.isfinite(traces))
    assert e_t <= tol
    if precision == "f64":
        assert e_p <= tol


CASES2D = {
    "halo0": lambda: ((400.0, 300.0), 0.3, 2000.0 * np.ones((41, 31)), [[200.0, 150.0]], [0.1],
                      10.0, [[100.0, 100.0]], dict(halo=0, freetop=False, check_ppw=False)),
    "rim_receivers": lambda: ((400.0, 300.0), 0.3, 2000.0 * np.ones((41, 31)), [[0.0, 150.0]],
                              [0.1], 10.0, [[0.0, 150.0], [400.0, 0.0], [10.0, 10.0]],
                              dict(halo=5, freetop=True, check_ppw=False)),
    "overlap": lambda: ((90.0, 80.0), 0.2, 2000.0 * np.ones((10, 9)), [[40.0, 40.0]], [0.1],
                        10.0, [[20.0, 30.0]], dict(halo=5, freetop=False, check_ppw=False)),
    "duplicates": lambda: ((400.0, 300.0), 0.3, 2000.0 * np.ones((41, 31)),
                           [[200.0, 150.0], [200.0, 150.0], [100.0, 50.0]], [0.1, 0.12, 0.1],
                           10.0, [[200.0, 150.0]], dict(halo=4, freetop=True, check_ppw=False)),
}


@pytest.mark.parametrize("name", sorted(CASES2D))
@pytest.mark.parametrize("precision,tol", [("f64", TOL64), ("f32", TOL32)])
def test_2d_edge_cases(pkg, oracle, ctx, name, precision, tol):
    s, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, CASES2D[name](), precision)
    assert cases.rel_l2(traces, traces_o) <= tol
    if precision == "f64":
        assert cases.rel_l2(pend, pend_o) <= tol


def test_plan_graph_eager_and_split_runs_agree(pkg, ctx):
    case = small3d(freetop=False)
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    kw = dict(kw)
    kw.pop("check_ppw")
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    s = pkg.prepare(lengths, lt, vel, srcs, recs, precision="f32", ppw=1e-9, **kw)
    plan = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"])
    nt = s["nt"]
    plan.run(graph=True)
    tr_g, p_g = plan.traces(), plan.field()
    plan.reset()
    plan.run(graph=False)
    tr_e, p_e = plan.traces(), plan.field()
    plan.reset()
    plan.run(7, graph=True)
    plan.run(nt // 2, graph=False)
    plan.run(graph=True)
    assert plan.step == nt
    tr_s, p_s = plan.traces(), plan.field()
    plan.close()
    np.testing.assert_array_equal(tr_g, tr_e)
    np.testing.assert_array_equal(p_g, p_e)
    np.testing.assert_array_equal(tr_g, tr_s)
    np.testing.assert_array_equal(p_g, p_s)


def test_launch_shapes_give_identical_results(pkg, ctx):
    """Every tile shape / z chunking computes the same numbers; sources and
    receivers (interior, rim, shared nodes) land in the right blocks."""
    srcs_pos = [[200.0, 80.0, 140.0], [200.0, 80.0, 140.0], [0.0, 50.0, 60.0],
                [390.0, 200.0, 10.0]]
    recs_pos = [[200.0, 80.0, 140.0], [0.0, 50.0, 60.0], [100.0, 330.0, 270.0],
                [310.0, 10.0, 20.0], [10.0, 20.0, 260.0]]
    lengths, lt, vel, sp, t0s, f0, rp, kw = small3d(srcs=srcs_pos, recs=recs_pos, freetop=False)
    kw = dict(kw)
    kw.pop("check_ppw")
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    for prec in ("f32", "f64"):
        s = pkg.prepare(lengths, lt, vel, srcs, recs, precision=prec, ppw=1e-9, **kw)
        plan = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                        s["posrecs"])
        plan.run()
        ref_t, ref_p = plan.traces(), plan.field()
        assert np.abs(ref_t).max() > 0
        shapes = ((4, 1, 1), (4, 7, 3), (8, 3, 10), (16, 5, 255), (16, 100, 7), (8, 26, 2))
        for ty, zc, bz in shapes:
            plan.set_launch(ty, zc, bz)
            plan.reset()
            plan.run()
            np.testing.assert_array_equal(plan.traces(), ref_t)
            np.testing.assert_array_equal(plan.field(), ref_p)
        plan.close()


def test_autotune_keeps_results(pkg, ctx):
    lengths, lt, vel, sp, t0s, f0, rp, kw = small3d(freetop=True)
    kw = dict(kw)
    kw.pop("check_ppw")
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    s = pkg.prepare(lengths, lt, vel, srcs, recs, precision="f32", ppw=1e-9, **kw)
    plan = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"])
    plan.run()
    ref = plan.traces()
    best = plan.autotune(5)
    assert best > 0 and plan.step == 0
    ty, zc, bz = plan.get_launch()
    assert ty in (4, 8, 16) and zc >= 1 and bz >= 1
    plan.run()
    np.testing.assert_array_equal(plan.traces(), ref)
    plan.close()


def test_forward_reuses_cached_plan(pkg, oracle, ctx):
    # two solves of one shape with different inputs: results follow the inputs
    a = run_both(pkg, oracle, ctx, small3d(seed=1), "f64")
    b = run_both(pkg, oracle, ctx, small3d(seed=2), "f64")
    for _, (pend, traces), (pend_o, traces_o) in (a, b):
        assert cases.rel_l2(traces, traces_o) <= TOL64
    assert cases.rel_l2(a[1][1], b[1][1]) > 1e-6


def _shot3d(d, freetop, srcs, recs, seed):
    """small3d's 40 x 34 x 28 grid with node spacing d."""
    nx, ny, nz = 40, 34, 28
    rng = np.random.default_rng(seed)
    vel = 2000.0 + 15.0 * np.arange(ny)[None, :, None] + 50.0 * rng.random((nx, ny, nz))
    L = ((nx - 1) * d, (ny - 1) * d, (nz - 1) * d)
    to_m = lambda pts: [[c * d for c in q] for q in pts]  # noqa: E731 (node index -> m)
    return (L, 0.2 * d / 10.0, vel, to_m(srcs), [0.05] * len(srcs), 12.0, to_m(recs),
            dict(halo=6, rcoef=1e-4, freetop=freetop, check_ppw=False))


def test_cached_graphs_follow_changed_inputs(pkg, oracle, ctx):
    """Shots of one shape in sequence through awc_forward, which keeps the
    plan and its CUDA graph while nothing the kernel parameters hold by value
    changes: the free top (live band sides), the spacing, and the
    source/receiver lists (with rim sources, so the rim list changes) vary
    from shot to shot; every result must follow its own inputs."""
    recs = [[2, 3, 3], [20, 3, 14], [37, 30, 24]]
    shots3d = [
        _shot3d(10.0, True, [[20, 8, 14]], recs, 1),
        _shot3d(10.0, False, [[20, 8, 14]], recs, 1),            # live sides change
        _shot3d(12.0, False, [[20, 8, 14]], recs, 1),            # spacing changes
        _shot3d(12.0, False, [[10, 0, 10], [21, 9, 13]], recs + [[10, 0, 10]], 2),  # rim
        _shot3d(12.0, False, [[21, 9, 13]] * 2, recs[:1], 3),    # back to no rim I/O
    ]
    shots2d = [((400.0, 300.0), 0.3, 2000.0 * np.ones((41, 31)), sp, [0.1] * len(sp), 10.0, rp,
                dict(halo=5, freetop=ft, check_ppw=False))
               for sp, rp, ft in (([[200.0, 150.0]], [[100.0, 100.0]], True),
                                  ([[200.0, 150.0]], [[100.0, 100.0]], False),
                                  ([[0.0, 150.0], [120.0, 80.0]], [[0.0, 150.0], [300.0, 20.0]],
                                   False),
                                  ([[120.0, 80.0]], [[300.0, 20.0]], True))]
    for case in shots3d + shots2d:
        for precision in ("f64", "f32"):
            _, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, case, precision)
            assert np.abs(traces_o).max() > 0
            if precision == "f64":
                assert cases.rel_l2(traces, traces_o) <= TOL64
                assert cases.rel_l2(pend, pend_o) <= TOL64
            else:
                assert cases.rel_l2(traces, traces_o) <= TOL32


def test_solve2D_api_golden(pkg):
    from acousticwavecpml_b200.Acoustic2D_CUDA import solve2D
    lengths, lt, vel, sp, t0s, f0, rp, kw = cases.ref_gradient()
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    pend = solve2D(*lengths, lt, vel, srcs, recs, **kw)
    assert cases.isapprox(pend, cases.golden("acoustic2D_gradient_freetop_halo20"))
    assert recs.seismograms.shape == (2504, 2)


def test_solve3D_api_analytic(pkg):
    """test/test3D_xPU.jl:12-59 through solve3D (FP64 and FP32)."""
    import test_oracle as T
    from acousticwavecpml_b200.Acoustic3D_CUDA import solve3D
    for precision in ("f64", "f32"):
        case = T.analytic_case_3d(20)
        lengths, lt, vel, sp, t0s, f0, rp, kw = case
        srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D], f0)
        recs = pkg.Receivers(rp)
        solve3D(*lengths, lt, vel, srcs, recs, precision=precision, **kw)
        s = pkg.prepare(lengths, lt, vel, srcs, recs, **kw)
        T.check_analytic(recs.seismograms[:, 0], s, case, 3)


def test_solve_errors(pkg):
    from acousticwavecpml_b200.Acoustic2D_CUDA import solve2D
    lengths, lt, vel, sp, t0s, f0, rp, kw = cases.ref_center(False)
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D], f0)
    with pytest.raises(AssertionError):
        solve2D(*lengths, lt, vel, srcs, pkg.Receivers([[-100.0, 5.0]]), **kw)
    with pytest.raises(NotImplementedError):
        solve2D(*lengths, lt, vel, srcs, pkg.Receivers(rp), do_vis=True, **kw)
    # the C ABI rejects an out-of-model position on its own
    s = pkg.prepare(lengths, lt, vel, srcs, pkg.Receivers(rp), **kw)
    bad = s["posrecs"].copy(order="F")
    bad[0, 0] = 0
    p = s["problem"]
    tr = np.zeros((p.nt, p.nrec), order="F")
    ctx = pkg.default_context(0)
    with pytest.raises(pkg.AwcInvalidArgument, match="not inside the model"):
        ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], bad, tr)
    # and stays usable afterwards
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr)
    assert np.abs(tr).max() > 0


@pytest.mark.parametrize("precision,tol", [("f64", TOL64), ("f32", TOL32)])
def test_config2_first_steps_vs_oracle(pkg, oracle, ctx, precision, tol):
    """The full-size headline grid (296 x 276 x 296), first 100 steps. The
    source peaks at t = 0 here (t0 = 0) so that the short run carries a
    wavefield well above FP32's range floor; the receivers are 5 nodes
    above the source and see it within 100 steps."""
    from acousticwavecpml_b200 import workloads as W
    w = W.config2(nt=100)
    w["t0s"] = [0.0]
    s, (pend, traces), (pend_o, traces_o) = run_both(pkg, oracle, ctx, _w2case(w), precision)
    e_t, e_p = cases.rel_l2(traces, traces_o), cases.rel_l2(pend, pend_o)
    print(f"config2 nt=100 {precision}: traces {e_t:.3e} field {e_p:.3e}")
    assert np.abs(traces_o).max() > 0
    assert e_p <= tol and e_t <= tol


# ---- 1D (the reference's solve1D) ------------------------------------------

def _analytic_1d_short(halo):
    """test/test1D.jl's line, run for 8 s: the pulses are still on the line,
    so the final field is not a residual far below the peak."""
    case = __import__("test_oracle").analytic_case_1d(halo)
    return case[:1] + (8.0,) + case[2:]


CASES1D = {
    "analytic_halo0": lambda: _analytic_1d_short(0),
    "analytic_halo20": lambda: _analytic_1d_short(20),
    # heterogeneous line, two sources (one on the Dirichlet end), receivers in
    # both bands and on a source node
    "layered": lambda: ((3990.0,), 1.5, np.where(np.arange(400) < 250, 1800.0, 2600.0),
                        [[1200.0], [0.0]], [0.08, 0.1], 12.0,
                        [[100.0], [3900.0], [1200.0], [2600.0]],
                        dict(halo=15, rcoef=1e-3, freetop=False)),
}


@pytest.mark.parametrize("name", sorted(CASES1D))
@pytest.mark.parametrize("precision,tol", [("f64", TOL64), ("f32", TOL32)])
def test_1d_vs_oracle(pkg, oracle, ctx, name, precision, tol):
    lengths, lt, vel, sp, t0s, f0, rp, kw = CASES1D[name]()
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    s = pkg.prepare(lengths, lt, vel, srcs, recs, precision=precision, **kw)
    p = s["problem"]
    assert p.ndim == 1
    traces = np.zeros((p.nt, p.nrec), order="F")
    pend = np.zeros(vel.shape, order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], traces, pend)
    so = oracle.setup(lengths, lt, vel, sp, t0s, f0, rp, **kw)
    pend_o, traces_o = oracle.forward_1d(so)
    e_t, e_p = cases.rel_l2(traces, traces_o), cases.rel_l2(pend, pend_o)
    print(f"1D {name} {precision}: traces rel-L2 {e_t:.3e}, field {e_p:.3e}")
    assert np.abs(traces_o).max() > 0
    assert e_t <= tol
    if precision == "f64":
        assert e_p <= tol


def test_solve1D_api_analytic(pkg):
    """test/test1D.jl:7-99 through solve1D (FP64 and FP32), halo 0 and 20."""
    import test_oracle as T
    from acousticwavecpml_b200.Acoustic1D import solve1D
    for halo in (0, 20):
        for precision in ("f64", "f32"):
            lengths, lt, vel, sp, t0s, f0, rp, kw = T.analytic_case_1d(halo)
            srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D], f0)
            recs = pkg.Receivers(rp)
            kw.pop("freetop")
            pend = solve1D(lengths[0], lt, vel, srcs, recs, precision=precision, verbose=False,
                           **kw)
            assert pend.shape == vel.shape
            s = pkg.prepare(lengths, lt, vel, srcs, recs, **kw)
            times, Gc = T.analytic_trace_1d(s["dt"], s["nt"], abs(sp[0][0] - rp[0][0]), 1.0,
                                            t0s[0], f0)
            err = T._trapz(times[1:], np.abs(recs.seismograms[:, 0] - Gc))
            assert err <= np.max(np.abs(Gc)) * 0.01 * lt, (halo, precision, err)


def test_1d_plan_snapshots_and_field(pkg, ctx):
    lengths, lt, vel, sp, t0s, f0, rp, kw = CASES1D["layered"]()
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    s = pkg.prepare(lengths, lt, vel, srcs, pkg.Receivers(rp), precision="f64", **kw)
    plan = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                    s["posrecs"])
    ref = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                   s["posrecs"])
    try:
        snaps = plan.run_snapshots(100, 25)
        for k in range(4):
            ref.run(25)
            np.testing.assert_array_equal(snaps[k], ref.field())
            assert snaps[k].shape == vel.shape
    finally:
        plan.close()
        ref.close()
