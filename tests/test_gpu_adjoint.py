"""Discrete adjoint (awc_misfit_gradient, awc_adjoint_sources) on the GPU.

* Dot-product test of the transpose of the source-to-trace map:
  <A s, r> = <s, Aᵀ r> to 1e-12 relative (FP64), 2D and 3D, with sources and
  receivers inside and outside the CPML bands.
* Gradient dJ/d(c²) against central finite differences of the FP64 oracle
  forward (eps = 1e-4 relative, 20 cells in 2D, 10 in 3D, dt fixed), 1e-6.
* The checkpoint interval does not change the gradient (bitwise); the FP32
  gradient follows the FP64 one (relative L2 <= 1e-4).
* The multi-shot call is bitwise the sum of the single-shot calls.
* A source on the Dirichlet rim: the gradient next to it against central
  differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def model2d(rng, nx=60, ny=50, d=10.0, freetop=True, halo=8):
    vel = 2000.0 + 8.0 * np.arange(ny)[None, :] + 100.0 * rng.random((nx, ny))
    L = ((nx - 1) * d, (ny - 1) * d)
    srcs = [[(nx // 2) * d, 6 * d], [3 * d, 20 * d]]  # one inside the x band
    recs = [[(i - 1) * d, 4 * d] for i in range(4, nx - 3, 5)] + [[(nx - 4) * d, (ny - 5) * d]]
    return L, vel, srcs, recs, dict(halo=halo, rcoef=1e-4, freetop=freetop)


def model3d(rng, n=(40, 36, 34), d=10.0, freetop=True, halo=6):
    nx, ny, nz = n
    vel = 2000.0 + 10.0 * np.arange(ny)[None, :, None] + 100.0 * rng.random(n)
    L = ((nx - 1) * d, (ny - 1) * d, (nz - 1) * d)
    srcs = [[(nx // 2) * d, 8 * d, (nz // 2) * d], [3 * d, 12 * d, 4 * d]]
    recs = [[(i - 1) * d, 3 * d, (k - 1) * d] for i in (4, nx // 2, nx - 3) for k in (5, nz - 4)]
    recs += [[(nx // 3) * d, (ny - 4) * d, (nz // 3) * d]]
    return L, vel, srcs, recs, dict(halo=halo, rcoef=1e-4, freetop=freetop)


def setup(pkg, L, vel, srcs, recs, kw, precision="f64", nt=None, lt=0.15, f0=12.0):
    S = pkg.Sources(srcs, [0.05] * len(srcs), [pkg.rickersource1D] * len(srcs), f0)
    R = pkg.Receivers(recs)
    return pkg.prepare(L, lt, vel, S, R, precision=precision, ppw=1e-9, nt=nt, **kw)


def traces_of(ctx, s):
    p = s["problem"]
    tr = np.zeros((p.nt, p.nrec), order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr)
    return tr


@pytest.mark.parametrize("dim,freetop", [(2, True), (2, False), (3, True), (3, False)])
def test_dot_product(pkg, ctx, dim, freetop):
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(3 + dim)
    L, vel, srcs, recs, kw = (model2d if dim == 2 else model3d)(rng, freetop=freetop)
    s = setup(pkg, L, vel, srcs, recs, kw)
    p = s["problem"]
    sa = rng.standard_normal((p.nt, p.nsrc))
    r = rng.standard_normal((p.nt, p.nrec))
    s2 = dict(s, dt2srctf=np.asfortranarray(sa))
    lhs = float(np.sum(traces_of(ctx, s2) * r))
    rhs = float(np.sum(sa * adjoint.adjoint_sources(s, r, ctx)))
    print(f"dot {dim}D freetop={freetop}: {lhs:.15e} {rhs:.15e}")
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


def _fd_cells(rng, vel, halo, n):
    shape = vel.shape
    cells = []
    vmax = vel.max()
    while len(cells) < n:
        c = tuple(int(rng.integers(1, m - 1)) for m in shape)
        if vel[c] < 0.99 * vmax and c not in cells:
            cells.append(c)
    return cells


@pytest.mark.parametrize("dim", [2, 3])
def test_gradient_vs_oracle_fd(pkg, oracle, ctx, dim):
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(11 + dim)
    L, vel, srcs, recs, kw = (model2d if dim == 2 else model3d)(rng)
    s = setup(pkg, L, vel, srcs, recs, kw)
    p = s["problem"]
    # observed data: a smoother model's traces
    s_obs = dict(s, vel=np.asfortranarray(np.full_like(vel, vel.mean())))
    obs = traces_of(ctx, s_obs)
    J, grad, traces = adjoint.misfit_gradient(s, obs, checkpoint_every=17, ctx=ctx)
    assert abs(J - 0.5 * np.sum((traces - obs) ** 2)) <= 1e-12 * J

    def oracle_J(v):
        so = oracle.setup(L, None, v, srcs, [0.05] * len(srcs), 12.0, recs, check_ppw=False,
                          dt=s["dt"], nt=p.nt, **kw)
        so["coeffs"] = s["coeffs"]  # fixed CPML profile (it depends on max(vel))
        _, tr = oracle.forward(so)
        return 0.5 * np.sum((tr - obs) ** 2)

    c2 = vel ** 2
    for cell in _fd_cells(rng, vel, kw["halo"], 20 if dim == 2 else 10):
        eps = 1e-4 * c2[cell]
        vp, vm = vel.copy(), vel.copy()
        vp[cell] = np.sqrt(c2[cell] + eps)
        vm[cell] = np.sqrt(c2[cell] - eps)
        fd = (oracle_J(vp) - oracle_J(vm)) / (2 * eps)
        print(f"{dim}D cell {cell}: adjoint {grad[cell]:.10e} fd {fd:.10e}")
        assert abs(grad[cell] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(grad).max())


def _small(dim, n, halo, freetop):
    """A grid too small for a band-free core (or just large enough)."""
    d = 10.0
    rng = np.random.default_rng(sum(n) + halo)
    shape = n[:dim]
    vel = 2000.0 + 100.0 * rng.random(shape)
    L = tuple((m - 1) * d for m in shape)
    c = [(m // 2) * d for m in shape]
    srcs = [c, [((shape[0] // 2) + 1) * d] + [2 * d] * (dim - 1)]
    recs = [[(i - 1) * d] + [3 * d] * (dim - 1) for i in (2, shape[0] // 2, shape[0] - 1)]
    return L, vel, srcs, recs, dict(halo=halo, rcoef=1e-4, freetop=freetop)


@pytest.mark.parametrize("dim,n,halo,freetop", [
    (3, (12, 13, 12), 4, False),   # the near-band zones meet: one generic shell box
    (3, (16, 15, 17), 4, True),    # a core of a few nodes
    (2, (12, 12, 1), 4, False),
    (3, (14, 12, 13), 0, False),   # no CPML: everything is core
])
def test_small_grids_dot_product_and_fd(pkg, oracle, ctx, dim, n, halo, freetop):
    """The adjoint's region split at its limits: the dot-product test and
    central differences of the FP64 oracle on a few cells."""
    from acousticwavecpml_b200 import adjoint
    L, vel, srcs, recs, kw = _small(dim, n, halo, freetop)
    s = setup(pkg, L, vel, srcs, recs, kw, lt=0.08)
    p = s["problem"]
    rng = np.random.default_rng(5)
    sa = rng.standard_normal((p.nt, p.nsrc))
    r = rng.standard_normal((p.nt, p.nrec))
    lhs = float(np.sum(traces_of(ctx, dict(s, dt2srctf=np.asfortranarray(sa))) * r))
    rhs = float(np.sum(sa * adjoint.adjoint_sources(s, r, ctx)))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))
    obs = traces_of(ctx, dict(s, vel=np.asfortranarray(np.full_like(vel, vel.mean()))))
    J, grad, _ = adjoint.misfit_gradient(s, obs, checkpoint_every=9, ctx=ctx)

    def oracle_J(v):
        so = oracle.setup(L, None, v, srcs, [0.05] * len(srcs), 12.0, recs, check_ppw=False,
                          dt=s["dt"], nt=p.nt, **kw)
        so["coeffs"] = s["coeffs"]
        _, tr = oracle.forward(so)
        return 0.5 * np.sum((tr - obs) ** 2)

    c2 = vel ** 2
    for cell in _fd_cells(rng, vel, halo, 6):
        eps = 1e-4 * c2[cell]
        vp, vm = vel.copy(), vel.copy()
        vp[cell] = np.sqrt(c2[cell] + eps)
        vm[cell] = np.sqrt(c2[cell] - eps)
        fd = (oracle_J(vp) - oracle_J(vm)) / (2 * eps)
        assert abs(grad[cell] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(grad).max()), cell


def test_gradient_with_rim_source_vs_oracle_fd(pkg, oracle, ctx):
    """A source on the Dirichlet rim (the free top) feeds the rim value of
    every pressure field, which the Laplacian of the interior nodes below it
    reads: the recomputed fields must carry it. Central differences of the
    FP64 oracle at the nodes next to that source and at random cells."""
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(31)
    L, vel, srcs, recs, kw = model2d(rng)
    srcs = srcs + [[20 * 10.0, 0.0]]  # node (20, 0): on the rim
    s = setup(pkg, L, vel, srcs, recs, kw)
    p = s["problem"]
    obs = traces_of(ctx, dict(s, vel=np.asfortranarray(np.full_like(vel, vel.mean()))))
    J, grad, _ = adjoint.misfit_gradient(s, obs, checkpoint_every=13, ctx=ctx)
    J1, grad1, _ = adjoint.misfit_gradient(s, obs, checkpoint_every=p.nt, ctx=ctx)
    assert J == J1 and np.array_equal(grad, grad1)

    def oracle_J(v):
        so = oracle.setup(L, None, v, srcs, [0.05] * len(srcs), 12.0, recs, check_ppw=False,
                          dt=s["dt"], nt=p.nt, **kw)
        so["coeffs"] = s["coeffs"]
        _, tr = oracle.forward(so)
        return 0.5 * np.sum((tr - obs) ** 2)

    c2 = vel ** 2
    cells = [(19, 1), (20, 1), (21, 1), (20, 2)] + _fd_cells(rng, vel, kw["halo"], 6)
    for cell in cells:
        eps = 1e-4 * c2[cell]
        vp, vm = vel.copy(), vel.copy()
        vp[cell] = np.sqrt(c2[cell] + eps)
        vm[cell] = np.sqrt(c2[cell] - eps)
        fd = (oracle_J(vp) - oracle_J(vm)) / (2 * eps)
        print(f"rim source, cell {cell}: adjoint {grad[cell]:.10e} fd {fd:.10e}")
        assert abs(grad[cell] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(grad).max())


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_checkpoint_interval_is_exact(pkg, ctx, precision):
    """Every checkpoint interval gives the same gradient, bit for bit, in
    both precisions."""
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(5)
    L, vel, srcs, recs, kw = model3d(rng, freetop=False)
    s = setup(pkg, L, vel, srcs, recs, kw, precision, nt=90)
    obs = np.zeros((90, s["problem"].nrec))
    ref = adjoint.misfit_gradient(s, obs, checkpoint_every=90, ctx=ctx)[1]
    for k in (1, 7, 50):
        g = adjoint.misfit_gradient(s, obs, checkpoint_every=k, ctx=ctx)[1]
        assert np.array_equal(g, ref), k
    assert np.abs(ref).max() > 0


@pytest.mark.parametrize("dim", [2, 3])
def test_fp32_gradient_follows_fp64(pkg, ctx, dim):
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(21 + dim)
    L, vel, srcs, recs, kw = (model2d if dim == 2 else model3d)(rng)
    s64 = setup(pkg, L, vel, srcs, recs, kw, "f64")
    s32 = setup(pkg, L, vel, srcs, recs, kw, "f32", nt=s64["nt"])
    s32["dt2srctf"] = s64["dt2srctf"]
    obs = traces_of(ctx, dict(s64, vel=np.asfortranarray(np.full_like(vel, vel.mean()))))
    J64, g64, _ = adjoint.misfit_gradient(s64, obs, 25, ctx)
    J32, g32, _ = adjoint.misfit_gradient(s32, obs, 25, ctx)
    e = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print(f"{dim}D fp32 gradient rel-L2 {e:.3e}, misfit {J32:.6e} vs {J64:.6e}")
    assert e <= 1e-4
    assert abs(J32 - J64) <= 1e-4 * J64


@pytest.mark.parametrize("dim,precision", [(2, "f64"), (3, "f32"), (3, "f64")])
def test_misfit_gradient_shots_is_the_sum_of_shots(pkg, ctx, dim, precision):
    """awc_misfit_gradient_shots (the model uploaded once, the gradients summed
    on the device) equals summing awc_misfit_gradient over the shots in order,
    bitwise, J and gradient; the shots move the two sources around the grid
    (band and core nodes), with observed data from another model."""
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(40 + dim)
    L, vel, srcs, recs, kw = (model2d if dim == 2 else model3d)(rng)
    d = 10.0
    n = vel.shape
    moves = [(0, 0), (5, -2), (-9, 3), (11, 7)]
    setups, obs = [], []
    true = np.asfortranarray(vel * (1.0 + 0.02 * rng.standard_normal(vel.shape)))
    for mx, my in moves:
        sh = [[min(max(c[0] + mx * d, 2 * d), (n[0] - 3) * d),
               min(max(c[1] + my * d, 2 * d), (n[1] - 3) * d)] + list(c[2:]) for c in srcs]
        s = setup(pkg, L, vel, sh, recs, kw, precision, nt=90)
        setups.append(s)
        obs.append(traces_of(ctx, dict(s, vel=true)))
    J_ref, g_ref = 0.0, np.zeros(vel.shape, order="F")
    for s, o in zip(setups, obs):
        j, g, _ = adjoint.misfit_gradient(s, o, 25, ctx)
        J_ref += j
        g_ref += g
    J, g = adjoint.misfit_gradient_shots(setups, obs, 25, ctx)
    assert J == J_ref
    assert np.array_equal(g, g_ref)
    assert np.abs(g_ref).max() > 0
    # one shot: the single-shot call's own result
    j0, g0, _ = adjoint.misfit_gradient(setups[2], obs[2], 25, ctx)
    J1, g1 = adjoint.misfit_gradient_shots(setups[2:3], obs[2:3], 25, ctx)
    assert J1 == j0 and np.array_equal(g1, g0)


@pytest.mark.parametrize("dim,precision", [(2, "f64"), (3, "f32")])
def test_misfit_gradient_shots_with_a_rim_source(pkg, ctx, dim, precision):
    """The middle one of three shots has a source on the Dirichlet rim: its
    recompute copies the fields instead of writing them in place, and the
    shots around it switch back. The sum must still be bitwise the sum of
    the single-shot calls."""
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(60 + dim)
    L, vel, srcs, recs, kw = (model2d if dim == 2 else model3d)(rng)
    d = 10.0
    rim = [20 * d, 0.0] + ([10 * d] if dim == 3 else [])
    inner = [srcs[0][0] + 2 * d] + list(srcs[0][1:])
    shots = [srcs + [inner], srcs + [rim], [inner] + srcs]
    true = np.asfortranarray(vel * (1.0 + 0.02 * rng.standard_normal(vel.shape)))
    setups = [setup(pkg, L, vel, sh, recs, kw, precision, nt=80) for sh in shots]
    obs = [traces_of(ctx, dict(s, vel=true)) for s in setups]
    J_ref, g_ref = 0.0, np.zeros(vel.shape, order="F")
    for s, o in zip(setups, obs):
        j, g, _ = adjoint.misfit_gradient(s, o, 15, ctx)
        J_ref += j
        g_ref += g
    J, g = adjoint.misfit_gradient_shots(setups, obs, 15, ctx)
    assert J == J_ref
    assert np.array_equal(g, g_ref)
    assert np.abs(g_ref).max() > 0


def test_misfit_gradient_shots_rejects_mixed_shots(pkg, ctx):
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(44)
    L, vel, srcs, recs, kw = model2d(rng)
    a = setup(pkg, L, vel, srcs, recs, kw, nt=60)
    b = setup(pkg, L, vel * 1.01, srcs, recs, kw, nt=60)
    o = np.zeros((60, a["problem"].nrec))
    with pytest.raises(ValueError):
        adjoint.misfit_gradient_shots([a, b], [o, o], 20, ctx)
    with pytest.raises(ValueError):
        adjoint.misfit_gradient_shots([a, a], [o], 20, ctx)


def test_torch_autograd_function(pkg, ctx):
    import torch
    from acousticwavecpml_b200 import adjoint
    rng = np.random.default_rng(8)
    L, vel, srcs, recs, kw = model2d(rng)
    s = setup(pkg, L, vel, srcs, recs, kw)
    obs = traces_of(ctx, dict(s, vel=np.asfortranarray(np.full_like(vel, vel.mean()))))
    c2 = torch.tensor(vel ** 2, dtype=torch.float64, requires_grad=True)
    J = adjoint.C2Misfit.apply(c2, s, obs, 20)
    J.backward()
    Jr, gr, _ = adjoint.misfit_gradient(s, obs, 20, ctx)
    assert abs(J.item() - Jr) <= 1e-12 * Jr
    assert np.allclose(c2.grad.numpy(), gr, rtol=0, atol=1e-12 * np.abs(gr).max())
