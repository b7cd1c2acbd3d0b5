"""Domain decomposition (awc_forward_decomposed), the reference's
multi-process strategy (src/shared/acoustic_3D_multixPU.jl:157-230,
acoustic_2D_multixPU.jl): subdomains along the last axis with a one-plane
halo exchange per step. Every node takes the same arithmetic as in the
undivided run, so traces and final fields must be bitwise equal to
awc_forward's. The subdomains run on one GPU here (one context repeated, or
several contexts on device 0); the exchange is the same peer copy that
crosses devices when the contexts sit on different GPUs."""
import numpy as np
import pytest

from test_gpu_forward import small3d

pytestmark = pytest.mark.gpu


def _setup(pkg, case, precision):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    kw = dict(kw)
    kw.pop("check_ppw", None)
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    return pkg.prepare(lengths, lt, vel, srcs, pkg.Receivers(rp), precision=precision,
                       ppw=1e-9, **kw)


def _both(pkg, ctxs, s):
    p = s["problem"]
    shape = s["vel"].shape
    tr = np.zeros((p.nt, p.nrec), order="F")
    pe = np.zeros(shape, order="F")
    ctxs[0].forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr, pe)
    trd = np.zeros((p.nt, p.nrec), order="F")
    ped = np.zeros(shape, order="F")
    pkg.core.forward_decomposed(ctxs, p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                                s["posrecs"], trd, ped)
    return tr, pe, trd, ped


def _case3d(nz, freetop):
    d = 10.0
    k_if = (nz - 2) // 2  # around the interface of two subdomains
    srcs = [[200.0, 80.0, k_if * d], [120.0, 90.0, (k_if + 1) * d], [0.0, 50.0, 60.0],
            [200.0, 80.0, 40.0]]
    recs = [[(i - 1) * d, 3 * d, (k - 1) * d] for i in (3, 20, 37) for k in (4, k_if, k_if + 1,
                                                                            k_if + 2, nz - 4)]
    recs += [[0.0, 50.0, 60.0], [100.0, 20.0, 0.0], [100.0, 20.0, (nz - 1) * d]]
    return small3d(n=(40, 34, nz), halo=6, freetop=freetop, srcs=srcs, recs=recs, lt=0.15)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("nsub,nz,freetop", [(2, 28, True), (3, 52, False), (2, 40, False)])
def test_decomposed_3d_equals_undivided(pkg, ctx, precision, nsub, nz, freetop):
    s = _setup(pkg, _case3d(nz, freetop), precision)
    tr, pe, trd, ped = _both(pkg, [ctx] * nsub, s)
    assert np.abs(tr).max() > 0
    np.testing.assert_array_equal(trd, tr)
    np.testing.assert_array_equal(ped, pe)


def test_decomposed_2d_depth_split_with_separate_contexts(pkg, ctx):
    """2D, split along depth (y) into three subdomains on three contexts of
    device 0 (their streams synchronise through events), free top, the
    reference gradient test's rim sources."""
    import cases
    lengths, lt, vel, sp, t0s, f0, rp, kw = cases.ref_gradient()
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp + [[5000.0, 2000.0], [5000.0, 2025.0], [100.0, 5900.0]])
    s = pkg.prepare(lengths, 1.5, vel, srcs, recs, precision="f64", **kw)
    ctxs = [ctx, pkg.Context(0), pkg.Context(0)]
    try:
        tr, pe, trd, ped = _both(pkg, ctxs, s)
    finally:
        for c in ctxs[1:]:
            c.close()
    assert np.abs(tr).max() > 0
    np.testing.assert_array_equal(trd, tr)
    np.testing.assert_array_equal(ped, pe)


def test_decomposed_refuses_thin_outer_subdomains(pkg, ctx):
    s = _setup(pkg, _case3d(28, True), "f32")
    p = s["problem"]
    tr = np.zeros((p.nt, p.nrec), order="F")
    with pytest.raises(pkg.AwcInvalidArgument, match="2 halo"):
        pkg.core.forward_decomposed([ctx] * 3, p, s["vel"], s["coeffs"], s["possrcs"],
                                    s["dt2srctf"], s["posrecs"], tr)
