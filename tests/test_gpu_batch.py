"""Batched 2D shots (awc_batch_*) on the GPU. Every shot of a batch must give
exactly the traces and final field of the same shot solved alone through
awc_forward (same kernels' arithmetic, so bitwise equal), for every launch
shape, with and without the CUDA graph and when run in pieces; sampled shots
are also checked against the FP64 oracle (relative L2 <= 1e-10 for the FP64
build, <= 1e-4 on traces for FP32)."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4
NT = 300


def _model(rng, nx, ny, d=10.0):
    vel = 2000.0 + 600.0 * rng.random((nx, ny))
    vel[:, ny // 2:] += 500.0
    return ((nx - 1) * d, (ny - 1) * d, np.asfortranarray(vel))


def small_batch(rng):
    """Three models of uneven size (one without a free top) and seven shots:
    uneven source/receiver counts, two sources on one node, sources and
    receivers on the Dirichlet rim and inside the CPML bands."""
    d = 10.0
    models = [_model(rng, 70, 50), _model(rng, 101, 64), _model(rng, 45, 77)]
    freetop = [True, True, False]
    shots = []
    for m, (lx, ly, _) in enumerate(models):
        for k in range(2 if m != 1 else 3):
            f0 = float(rng.uniform(8.0, 13.0))
            sx = (k + 1) * lx / (4 if m != 1 else 5)
            sp = [[sx, 3 * d]]
            if m == 1 and k == 0:
                sp = [[sx, 3 * d], [sx, 3 * d], [lx / 2, ly / 2]]     # two on one node
            if m == 0 and k == 1:
                sp = [[lx / 2, 0.0], [2 * d, ly / 3]]                 # rim and x band
            rp = [[x, 2 * d] for x in np.linspace(0.0, lx, 9)]        # includes rim nodes
            if m == 2:
                rp += [[lx / 2, ly - d], [lx - d, ly / 2]]
            t0s = [float(rng.uniform(0.9, 1.4)) / f0 for _ in sp]
            shots.append((m, sp, t0s, f0, rp))
    return models, freetop, shots


def prepared(pkg, models, freetop, shots, precision, nt=NT, halo=8):
    setups, probs, vels = [], [], []
    for m, sp, t0s, f0, rp in shots:
        lx, ly, vel = models[m]
        srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(sp), f0)
        setups.append(pkg.prepare((lx, ly), None, vel, srcs, pkg.Receivers(rp), halo=halo,
                                  rcoef=1e-4, freetop=freetop[m], precision=precision, nt=nt))
    for m, (lx, ly, vel) in enumerate(models):
        p = next(s["problem"] for s, sh in zip(setups, shots) if sh[0] == m)
        probs.append(pkg.Problem(ndim=2, precision=p.precision, nx=p.nx, ny=p.ny, nz=1,
                                 halo=p.halo, freetop=p.freetop, dx=p.dx, dy=p.dy, dz=1.0,
                                 dt=p.dt, nt=p.nt, nsrc=0, nrec=0))
        vels.append(vel)
    return probs, vels, setups, [sh[0] for sh in shots]


def single(ctx, s):
    p = s["problem"]
    traces = np.zeros((p.nt, p.nrec), order="F")
    pend = np.zeros(s["vel"].shape, order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], traces, pend)
    return traces, pend


@pytest.fixture(scope="module", params=["f64", "f32"])
def batch_case(request, pkg, ctx):
    rng = np.random.default_rng(7)
    models, freetop, shots = small_batch(rng)
    probs, vels, setups, idx = prepared(pkg, models, freetop, shots, request.param)
    refs = [single(ctx, s) for s in setups]
    return request.param, models, freetop, shots, probs, vels, setups, idx, refs


def _all_equal(b, refs):
    for k, (tr, pe) in enumerate(refs):
        t = b.traces(k)
        f = b.field(k)
        assert np.array_equal(t, tr), (k, cases.rel_l2(t, tr))
        assert np.array_equal(f, pe), (k, cases.rel_l2(f, pe))


def test_batch_equals_single_shots(pkg, ctx, batch_case):
    _, _, _, _, probs, vels, setups, idx, refs = batch_case
    b = pkg.Batch(ctx, probs, vels, setups, idx)
    b.run()
    assert b.step == NT
    _all_equal(b, refs)
    b.close()


@pytest.mark.parametrize("ty,bps", [(4, 4), (8, 8), (16, 32), (32, 1), (64, 2), (64, 16)])
def test_batch_launch_shapes(pkg, ctx, batch_case, ty, bps):
    _, _, _, _, probs, vels, setups, idx, refs = batch_case
    b = pkg.Batch(ctx, probs, vels, setups, idx)
    b.set_launch(ty, bps)
    assert b.get_launch() == (ty, bps)
    b.run()
    _all_equal(b, refs)
    b.close()


def test_batch_pieces_graph_and_reset(pkg, ctx, batch_case):
    _, _, _, _, probs, vels, setups, idx, refs = batch_case
    b = pkg.Batch(ctx, probs, vels, setups, idx)
    b.run(1, graph=False)
    b.run(120)
    b.run(NT - 121, graph=False)
    assert b.step == NT
    _all_equal(b, refs)
    b.reset()
    assert b.step == 0
    b.run()
    _all_equal(b, refs)
    b.close()


def test_batch_autotune(pkg, ctx, batch_case):
    _, _, _, _, probs, vels, setups, idx, refs = batch_case
    b = pkg.Batch(ctx, probs, vels, setups, idx)
    ms = b.autotune(5)
    assert ms > 0.0
    ty, bps = b.get_launch()
    assert ty in (4, 8, 16, 32, 64) and bps >= 1
    assert b.step == 0
    b.run()
    _all_equal(b, refs)
    b.close()


def test_batch_vs_oracle(pkg, oracle, ctx, batch_case):
    precision, models, freetop, shots, probs, vels, setups, idx, refs = batch_case
    b = pkg.Batch(ctx, probs, vels, setups, idx)
    b.run()
    for k in (0, 2, 5):
        m, sp, t0s, f0, rp = shots[k]
        lx, ly, vel = models[m]
        so = oracle.setup((lx, ly), None, vel, sp, t0s, f0, rp, halo=8, rcoef=1e-4,
                          freetop=freetop[m], dt=setups[k]["dt"], nt=NT)
        pend_o, traces_o = oracle.forward(so)
        e = cases.rel_l2(b.traces(k), traces_o)
        print(f"batch {precision} shot {k}: traces rel-L2 {e:.3e}")
        if precision == "f64":
            assert e <= TOL64
            assert cases.rel_l2(b.field(k), pend_o) <= TOL64
        else:
            assert e <= TOL32
    b.close()


def test_forward_batch_entry(pkg, ctx, batch_case):
    """awc_forward_batch: the one-call form (create, autotune, run, traces,
    destroy)."""
    _, _, _, _, probs, vels, setups, idx, refs = batch_case
    outs = pkg.forward_batch(ctx, probs, vels, setups, idx)
    for k, (tr, _) in enumerate(refs):
        assert np.array_equal(outs[k], tr), k


def test_solve2D_batch_config3_sampled(pkg, oracle, ctx):
    """The batched-shot workload (6 layered models, 96 shots) for its first
    400 steps: sampled shots vs the single-shot solve, and the smallest
    model's first shot vs the oracle."""
    from acousticwavecpml_b200 import workloads as W
    w = W.config3(nt=400)
    shots = W.batch_shots(pkg, w)
    pkg.solve2D_batch(w["models"], shots, **w["kwargs"])
    kw = dict(w["kwargs"])
    for k in (0, 23, 40, 57, 74, 95):
        m, srcs, recs = shots[k]
        lx, ly, vel = w["models"][m]
        s = pkg.prepare((lx, ly), None, vel, srcs, pkg.Receivers(recs.positions),
                        precision="f32", **kw)
        tr, _ = single(ctx, s)
        assert np.array_equal(recs.seismograms, tr), k
    sh = w["shots"][0]
    lx, ly, vel = w["models"][0]
    dt = pkg.prepare((lx, ly), None, vel, shots[0][1], shots[0][2], **kw)["dt"]
    so = oracle.setup((lx, ly), None, vel, sh["src_pos"], sh["t0s"], sh["f0"], sh["rec_pos"],
                      halo=kw["halo"], rcoef=kw["rcoef"], freetop=True, dt=dt, nt=kw["nt"])
    _, traces_o = oracle.forward(so)
    e = cases.rel_l2(shots[0][2].seismograms, traces_o)
    print(f"config3 shot 0 f32 traces rel-L2 vs oracle {e:.3e}")
    assert e <= TOL32


def test_batch_rejects_bad_input(pkg, ctx, batch_case):
    _, _, _, _, probs, vels, setups, idx, _ = batch_case
    with pytest.raises(pkg.AwcInvalidArgument):
        pkg.Batch(ctx, probs, vels, setups, [len(probs)] + idx[1:])
    bad = [pkg.Problem.from_buffer_copy(p) for p in probs]
    bad[1].nt = NT + 1
    with pytest.raises(pkg.AwcInvalidArgument):
        pkg.Batch(ctx, bad, vels, setups, idx)
    s0 = dict(setups[0])
    pos = np.array(s0["possrcs"], order="F")
    pos[0, 0] = probs[idx[0]].nx + 1
    s0["possrcs"] = pos
    with pytest.raises(pkg.AwcInvalidArgument, match="source"):
        pkg.Batch(ctx, probs, vels, [s0] + setups[1:], idx)
