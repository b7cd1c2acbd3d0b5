"""Host side of the multi-shot gradient (no GPU): the stacked inputs that
awc_misfit_gradient_shots reads (per-shot blocks at the strides its header
states) and the checks that reject shots of different models."""
import numpy as np
import pytest


def _setups(pkg, n=3, vel_scale=None, recs_shift=0):
    d = 10.0
    shape = (40, 34)
    rng = np.random.default_rng(9)
    vel = 2000.0 + 100.0 * rng.random(shape)
    L = tuple((m - 1) * d for m in shape)
    recs = [[(4 + 3 * i + recs_shift) * d, 4 * d] for i in range(6)]
    out = []
    for s in range(n):
        v = vel * (vel_scale[s] if vel_scale else 1.0)
        srcs = [[(10 + 3 * s) * d, 6 * d], [(25 - 2 * s) * d, 12 * d]]
        S = pkg.Sources(srcs, [0.05, 0.06], [pkg.rickersource1D] * 2, 12.0)
        R = pkg.Receivers(recs)
        out.append(pkg.prepare(L, None, v, S, R, halo=6, ppw=1e-9, precision="f32", nt=40,
                               dt=1e-3))
    return out


def test_stacked_blocks_follow_the_header_strides(pkg):
    from acousticwavecpml_b200 import adjoint
    setups = _setups(pkg)
    p = setups[0]["problem"]
    rng = np.random.default_rng(1)
    observed = [rng.standard_normal((p.nt, p.nrec)) for _ in setups]
    pos, stf, obs = adjoint.stack_shots(setups, observed)
    assert pos.dtype == np.int64 and pos.flags.f_contiguous
    assert stf.flags.f_contiguous and obs.flags.f_contiguous
    fp, fs, fo = (a.ravel(order="K") for a in (pos, stf, obs))
    bp, bs, bo = p.nsrc * 2, p.nt * p.nsrc, p.nt * p.nrec
    for s, st in enumerate(setups):
        assert np.array_equal(fp[s * bp:(s + 1) * bp], np.asarray(st["possrcs"]).ravel(order="F"))
        assert np.array_equal(fs[s * bs:(s + 1) * bs], np.asarray(st["dt2srctf"]).ravel(order="F"))
        assert np.array_equal(fo[s * bo:(s + 1) * bo], observed[s].ravel(order="F"))
    # the sources differ from shot to shot
    assert not np.array_equal(fp[:bp], fp[bp:2 * bp])


def test_stacked_observed_is_used_in_place(pkg):
    from acousticwavecpml_b200 import adjoint
    setups = _setups(pkg)
    p = setups[0]["problem"]
    obs3 = np.asfortranarray(np.ones((p.nt, p.nrec, len(setups))))
    _, _, obs = adjoint.stack_shots(setups, obs3)
    assert np.shares_memory(obs, obs3)


def test_shots_of_different_models_are_rejected(pkg):
    from acousticwavecpml_b200 import adjoint
    base = _setups(pkg)
    p = base[0]["problem"]
    obs = [np.zeros((p.nt, p.nrec))] * 3
    with pytest.raises(ValueError):  # another velocity model
        adjoint.stack_shots(_setups(pkg, vel_scale=[1.0, 1.0, 0.999]), obs)
    other_recs = _setups(pkg, recs_shift=1)
    with pytest.raises(ValueError):  # other receivers
        adjoint.stack_shots([base[0], other_recs[1]], obs[:2])
    with pytest.raises(ValueError):  # one observed array short
        adjoint.stack_shots(base, obs[:2])
    with pytest.raises(ValueError):  # wrong trace shape
        adjoint.stack_shots(base, [np.zeros((p.nt + 1, p.nrec))] * 3)
    with pytest.raises(ValueError):
        adjoint.stack_shots([], [])
