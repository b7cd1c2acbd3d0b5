"""The benchmark configurations at their full sizes and lengths against the
FP64 oracle (the errors are also printed, one line per configuration).

Config 1: 2D FP64 and FP32, 241 x 241, nt = 1000 (test_gpu_forward.py).
Config 2: 3D FP64 and FP32, 296 x 276 x 296, nt = 2000: one oracle run, the
  FP64 build within 1e-10 on traces and final field, the FP32 build within
  1e-4 on traces.
Config 3: the 96 batched FP32 shots at nt = 3000, the first shot of each of
  the 6 models against the oracle (1e-4 on traces).
Config 4: 3D 232 x 212 x 232, nt = 1500, checkpoints every 50 steps:
  dot-product test of the adjoint (1e-12, FP64), the gradient of shot 0
  against central differences (eps = 1e-4 relative and eps/2, combined to
  cancel the O(eps²) term; 20 cells; dt and the CPML profile fixed) of the
  FP64 forward, which itself matches the oracle within 1e-10, the FP32
  gradient of two shots against the FP64 one, and the FP32 adjoint on the FP64
  residual against the FP64 gradient (1e-4).
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4


def _case(w):
    return (w["lengths"], w["lt"], w["vel"], w["src_pos"], w["t0s"], w["f0"], w["rec_pos"],
            w["kwargs"])


def _forward(pkg, ctx, s):
    p = s["problem"]
    tr = np.zeros((p.nt, p.nrec), order="F")
    pe = np.zeros(s["vel"].shape, order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr, pe)
    return tr, pe


@pytest.fixture(scope="module")
def config2_oracle(oracle):
    from acousticwavecpml_b200 import workloads as W
    w = W.config2()
    so = oracle.setup(w["lengths"], w["lt"], w["vel"], w["src_pos"], w["t0s"], w["f0"],
                      w["rec_pos"], **w["kwargs"])
    pend, traces = oracle.forward(so)
    return w, pend, traces


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_config2_full_length_vs_oracle(pkg, ctx, config2_oracle, precision):
    w, pend_o, traces_o = config2_oracle
    srcs = pkg.Sources(w["src_pos"], w["t0s"], [pkg.rickersource1D], w["f0"])
    recs = pkg.Receivers(w["rec_pos"])
    s = pkg.prepare(w["lengths"], w["lt"], w["vel"], srcs, recs, precision=precision,
                    **w["kwargs"])
    assert s["nt"] == 2000
    tr, pe = _forward(pkg, ctx, s)
    e_t, e_p = cases.rel_l2(tr, traces_o), cases.rel_l2(pe, pend_o)
    print(f"config2 296x276x296 nt=2000 {precision}: traces rel-L2 {e_t:.3e}, "
          f"final field {e_p:.3e} vs the FP64 oracle")
    assert np.abs(traces_o).max() > 0
    if precision == "f64":
        assert e_t <= TOL64 and e_p <= TOL64
    else:
        assert e_t <= TOL32


def test_config3_full_length_vs_oracle(pkg, oracle, ctx):
    from acousticwavecpml_b200 import workloads as W
    w = W.config3()
    assert w["kwargs"]["nt"] == 3000
    shots = W.batch_shots(pkg, w)
    pkg.solve2D_batch(w["models"], shots, **w["kwargs"])
    kw = w["kwargs"]
    firsts = {}
    for k, sh in enumerate(w["shots"]):
        firsts.setdefault(sh["model"], k)
    for m, k in sorted(firsts.items()):
        sh = w["shots"][k]
        lx, ly, vel = w["models"][m]
        dt = pkg.prepare((lx, ly), None, vel, shots[k][1], pkg.Receivers(sh["rec_pos"]),
                         **kw)["dt"]
        so = oracle.setup((lx, ly), None, vel, sh["src_pos"], sh["t0s"], sh["f0"],
                          sh["rec_pos"], halo=kw["halo"], rcoef=kw["rcoef"], freetop=True,
                          dt=dt, nt=kw["nt"])
        _, traces_o = oracle.forward(so)
        e = cases.rel_l2(shots[k][2].seismograms, traces_o)
        print(f"config3 model {m} ({vel.shape[0]}x{vel.shape[1]}) shot {k} nt=3000 f32: "
              f"traces rel-L2 {e:.3e} vs the FP64 oracle")
        assert np.abs(traces_o).max() > 0
        assert e <= TOL32


@pytest.fixture(scope="module")
def config4(pkg):
    from acousticwavecpml_b200 import workloads as W
    w = W.config4()
    kw = dict(w["kwargs"])
    recs = w["rec_pos"]

    def setup(vel, shot, precision):
        srcs = pkg.Sources(w["shots"][shot], w["t0s"], [pkg.rickersource1D], w["f0"])
        return pkg.prepare(w["lengths"], None, vel, srcs, pkg.Receivers(recs),
                           precision=precision, **kw)

    return w, setup


def test_config4_dot_product_full_size(pkg, ctx, config4):
    from acousticwavecpml_b200 import adjoint
    w, setup = config4
    s = setup(w["init"], 0, "f64")
    p = s["problem"]
    rng = np.random.default_rng(41)
    sa = rng.standard_normal((p.nt, p.nsrc))
    r = rng.standard_normal((p.nt, p.nrec))
    tr, _ = _forward(pkg, ctx, dict(s, dt2srctf=np.asfortranarray(sa)))
    lhs = float(np.sum(tr * r))
    rhs = float(np.sum(sa * adjoint.adjoint_sources(s, r, ctx)))
    print(f"config4 232x212x232 nt=1500 dot product: {lhs:.15e} {rhs:.15e} "
          f"rel {abs(lhs - rhs) / max(abs(lhs), abs(rhs)):.2e}")
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


def test_config4_gradient_vs_central_differences(pkg, oracle, ctx, config4):
    from acousticwavecpml_b200 import adjoint
    w, setup = config4
    s_obs = setup(w["true"], 0, "f64")
    obs, _ = _forward(pkg, ctx, s_obs)
    s = setup(w["init"], 0, "f64")
    s["dt2srctf"] = s_obs["dt2srctf"]
    s["coeffs"] = s_obs["coeffs"]
    p = s["problem"]
    # the FP64 forward of this set-up is the oracle's within 1e-10
    so = oracle.setup(w["lengths"], None, w["init"], w["shots"][0], w["t0s"], w["f0"],
                      w["rec_pos"], check_ppw=False, **w["kwargs"])
    so["coeffs"] = s["coeffs"]
    _, tr_o = oracle.forward(so)
    tr, _ = _forward(pkg, ctx, s)
    e_fwd = cases.rel_l2(tr, tr_o)
    print(f"config4 shot 0 FP64 forward traces rel-L2 vs the oracle {e_fwd:.3e}")
    assert e_fwd <= TOL64
    J, grad, _ = adjoint.misfit_gradient(s, obs, checkpoint_every=50, ctx=ctx)
    assert J > 0

    def J_of(vel):
        t, _ = _forward(pkg, ctx, dict(s, vel=np.asfortranarray(vel)))
        return 0.5 * float(np.sum((t - obs) ** 2))

    vel = np.asarray(w["init"], dtype=np.float64)
    c2 = vel ** 2
    rng = np.random.default_rng(99)
    h = w["kwargs"]["halo"]
    interior = tuple(slice(1, n - 1) for n in vel.shape)
    g_in = np.abs(grad[interior])
    # 10 cells where the gradient is largest, 10 random interior cells
    flat = np.argsort(g_in, axis=None)[::-1][:2000:200]
    cells = [tuple(int(i) + 1 for i in np.unravel_index(f, g_in.shape)) for f in flat]
    while len(cells) < 20:
        c = tuple(int(rng.integers(1, n - 1)) for n in vel.shape)
        if c not in cells and vel[c] < 0.99 * vel.max():
            cells.append(c)
    gmax = np.abs(grad).max()
    worst = 0.0

    def central(cell, eps):
        vp, vm = vel.copy(), vel.copy()
        vp[cell] = np.sqrt(c2[cell] + eps)
        vm[cell] = np.sqrt(c2[cell] - eps)
        return (J_of(vp) - J_of(vm)) / (2 * eps)

    for cell in cells:
        # central differences at eps and eps/2 (eps = 1e-4 c²), combined to
        # cancel their O(eps²) term, which is not small next to a derivative
        # a few hundred times below the largest
        eps = 1e-4 * c2[cell]
        fd = (4.0 * central(cell, eps / 2) - central(cell, eps)) / 3.0
        err = abs(grad[cell] - fd) / max(abs(fd), 1e-3 * gmax)
        worst = max(worst, err)
        print(f"config4 cell {cell} (halo {h}): adjoint {grad[cell]:.10e} fd {fd:.10e} "
              f"rel {err:.2e}")
        assert err <= 1e-6
    print(f"config4 gradient vs central differences, 20 cells: worst {worst:.2e}")


def test_config4_fp32_gradient_two_shots(pkg, ctx, config4):
    """Each precision against observed data of its own precision (the true
    model's traces): against FP64 data the FP32 residual would also carry
    the FP32 rounding of the direct wave, whose imprint near the source is
    not a property of the gradient computation."""
    from acousticwavecpml_b200 import adjoint
    w, setup = config4
    g = {}
    J = {}
    for prec in ("f64", "f32"):
        g[prec] = np.zeros(w["init"].shape)
        J[prec] = 0.0
        for shot in (0, 5):
            s_obs = setup(w["true"], shot, prec)
            obs, _ = _forward(pkg, ctx, s_obs)
            s = setup(w["init"], shot, prec)
            s["dt2srctf"] = s_obs["dt2srctf"]
            s["coeffs"] = s_obs["coeffs"]
            j, gr, _ = adjoint.misfit_gradient(s, obs, 50, ctx)
            g[prec] += gr
            J[prec] += j
    e = cases.rel_l2(g["f32"], g["f64"])
    print(f"config4 two shots: FP32 vs FP64 gradient rel-L2 {e:.3e}, misfit "
          f"{J['f32']:.8e} vs {J['f64']:.8e}")
    assert e <= 3e-4
    assert abs(J["f32"] - J["f64"]) <= 1e-4 * J["f64"]


def test_config4_fp32_adjoint_on_the_fp64_residual(pkg, ctx, config4):
    """The FP32 gradient's difference from the FP64 one comes from the
    residual: FP32 traces differ from FP64 ones by about 3e-7, but the
    residual (traces - observed, about 1e-3 of the traces for this blob) then
    differs by about 3e-4. Given the FP64 residual, the FP32 adjoint and
    gradient accumulation match the FP64 gradient within 1e-4."""
    from acousticwavecpml_b200 import adjoint
    w, setup = config4
    out = {}
    for prec in ("f64", "f32"):
        s_obs = setup(w["true"], 0, prec)
        obs, _ = _forward(pkg, ctx, s_obs)
        s = setup(w["init"], 0, prec)
        s["dt2srctf"] = s_obs["dt2srctf"]
        s["coeffs"] = s_obs["coeffs"]
        out[prec] = (s, obs) + tuple(adjoint.misfit_gradient(s, obs, 50, ctx))
    s64, obs64, J64, g64, tr64 = out["f64"]
    s32, obs32, J32, g32, tr32 = out["f32"]
    # observed data for the FP32 run such that its residual is the FP64 one
    inj = np.asfortranarray(tr32 - (tr64 - obs64))
    J, g, _ = adjoint.misfit_gradient(s32, inj, 50, ctx)
    e_own = cases.rel_l2(g32, g64)
    e_res = cases.rel_l2((tr32 - obs32), (tr64 - obs64))
    e = cases.rel_l2(g, g64)
    print(f"config4 shot 0: FP32 gradient vs FP64 {e_own:.3e} (residuals differ by {e_res:.3e}); "
          f"FP32 adjoint on the FP64 residual vs FP64 {e:.3e}")
    assert e <= 1e-4
    assert abs(J - J64) <= 1e-10 * J64

