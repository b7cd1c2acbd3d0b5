"""Host side of batched shots: the awc_shot struct layout, the batched-shot
workload builder and the per-shot set-up (no GPU)."""
import ctypes

import numpy as np


def test_shot_struct_layout(pkg):
    from acousticwavecpml_b200 import _lib
    S = _lib.Shot
    assert S.model.offset == 0 and S.nsrc.offset == 4 and S.nrec.offset == 8
    ptr = ctypes.sizeof(ctypes.c_void_p)
    assert S.coeffs.offset == 16 and S.posrecs.offset == 16 + 3 * ptr
    assert ctypes.sizeof(S) == 16 + 4 * ptr


def test_config3_workload(pkg):
    from acousticwavecpml_b200 import workloads as W
    w = W.config3(nt=10)
    assert len(w["models"]) == 6 and len(w["shots"]) == 96
    sizes = [m[2].shape for m in w["models"]]
    assert sizes == [(ix + 40, iy + 20) for ix, iy in W.CONFIG3_INTERIORS]
    for lx, ly, vel in w["models"]:
        assert vel.flags.f_contiguous
        assert 1400.0 < vel.min() and vel.max() < 4700.0
        col = np.median(vel, axis=0)
        assert np.all(np.diff(col) >= -100.0)  # velocity grows with depth
    f0 = np.array([s["f0"] for s in w["shots"]])
    assert np.all((f0 >= 10.0) & (f0 <= 20.0))
    assert [s["model"] for s in w["shots"]] == sorted(m for m in range(6) for _ in range(16))
    w2 = W.config3(nt=10)
    assert all(np.array_equal(a[2], b[2]) for a, b in zip(w["models"], w2["models"]))


def test_prepare_batch_mapping(pkg):
    from acousticwavecpml_b200 import workloads as W
    w = W.config3(nt=50, shots_per_model=2, interiors=((64, 32), (96, 48), (80, 40)))
    shots = [s for s in W.batch_shots(pkg, w) if s[0] != 1]  # model 1 unused
    probs, vels, setups, idx = pkg.prepare_batch(w["models"], shots, **w["kwargs"])
    assert len(probs) == 2 and idx == [0, 0, 1, 1]
    assert (probs[0].nx, probs[0].ny) == (104, 52) and (probs[1].nx, probs[1].ny) == (120, 60)
    assert all(p.nt == 50 and p.nsrc == 0 and p.nrec == 0 for p in probs)
    for k, s in enumerate(setups):
        p = s["problem"]
        assert (p.nx, p.ny) == (probs[idx[k]].nx, probs[idx[k]].ny)
        assert p.dt == probs[idx[k]].dt
        assert np.all(s["possrcs"][:, 1] == 3)      # depth node j = 3
        assert np.all(s["posrecs"][:, 1] == 3)
        assert s["posrecs"][0, 0] == 21 and np.all(np.diff(s["posrecs"][:, 0]) == 4)
    # CPML coefficients depend on each shot's f0 (alpha_max = pi f0)
    assert not np.array_equal(setups[0]["coeffs"], setups[1]["coeffs"])
