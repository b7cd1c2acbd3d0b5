"""Snapshot output (awc_plan_run_snapshots and solve3D's do_save), the
reference's do_save branch (src/shared/acoustic_3D_xPU.jl:375-379,479-498):
the field after every step it with it % nsave == 0. Each snapshot must equal
awc_plan_field read at that step (bitwise), and a run with snapshots must
leave the same traces and final field as one without."""
import glob
import os

import numpy as np
import pytest

from test_gpu_forward import small3d

pytestmark = pytest.mark.gpu


def _plan(pkg, ctx, case, precision="f32"):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    kw = dict(kw)
    kw.pop("check_ppw", None)
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    s = pkg.prepare(lengths, lt, vel, srcs, recs, precision=precision, ppw=1e-9, **kw)
    return s, ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                       s["posrecs"])


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_snapshots_equal_fields_at_those_steps(pkg, ctx, precision):
    s, ref = _plan(pkg, ctx, small3d(freetop=True), precision)
    s2, plan = _plan(pkg, ctx, small3d(freetop=True), precision)
    try:
        nt, nsave = s["nt"], 6
        expect = []
        while ref.step + nsave <= nt:
            ref.run(nsave)
            expect.append(ref.field())
        ref.run()
        got = []
        # uneven pieces: 4 snapshots, then 1, then the rest
        got += plan.run_snapshots(4 * nsave + 3, nsave)
        got += plan.run_snapshots(nsave, nsave)
        while plan.step < nt:
            got += plan.run_snapshots(5 * nsave, nsave)
        assert len(got) == nt // nsave == len(expect)
        for a, b in zip(got, expect):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(plan.traces(), ref.traces())
        np.testing.assert_array_equal(plan.field(), ref.field())
        assert np.abs(expect[-1]).max() > 0
    finally:
        ref.close()
        plan.close()


def test_snapshot_buffer_too_small_is_refused(pkg, ctx):
    s, plan = _plan(pkg, ctx, small3d(), "f32")
    try:
        buf = np.zeros((2,) + s["vel"].shape[::-1])
        with pytest.raises(pkg.AwcInvalidArgument, match="snapshots"):
            plan.run_snapshots(30, 5, buf)
        assert plan.step == 0  # nothing ran
        assert len(plan.run_snapshots(10, 5, buf)) == 2
    finally:
        plan.close()


def test_solve3D_do_save_writes_the_reference_datasets(pkg, ctx, tmp_path):
    from acousticwavecpml_b200.Acoustic3D_CUDA import solve3D
    lengths, lt, vel, sp, t0s, f0, rp, kw = small3d(freetop=True)
    kw = dict(kw)
    kw.pop("check_ppw", None)

    def srcs_recs():
        return pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0), pkg.Receivers(rp)

    S, R = srcs_recs()
    pend = solve3D(*lengths, lt, vel, S, R, ppw=1e-9, precision="f32", verbose=False, **kw)
    S2, R2 = srcs_recs()
    pend2 = solve3D(*lengths, lt, vel, S2, R2, ppw=1e-9, precision="f32", verbose=False,
                    do_save=True, nsave=7, save_name="snap", save_dir=str(tmp_path), **kw)
    np.testing.assert_array_equal(pend2, pend)
    np.testing.assert_array_equal(R2.seismograms, R.seismograms)
    nt = R.seismograms.shape[0]
    files = sorted(glob.glob(os.path.join(str(tmp_path), "snap_it*")))
    assert len(files) == nt // 7
    # the snapshot after step 14 is the field of a 14-step run
    s, plan = _plan(pkg, ctx, small3d(freetop=True), "f32")
    try:
        plan.run(14)
        ref = plan.field()
    finally:
        plan.close()
    path = [f for f in files if os.path.basename(f).startswith("snap_it14.")][0]
    if path.endswith(".npz"):
        d = np.load(path)
        keys = set(d.files)
        pcur = d["pcur"]
    else:
        import h5py
        with h5py.File(path, "r") as d:
            keys = set(d.keys())
            pcur = d["pcur"][()]
    assert {"lx", "ly", "lz", "halo", "pcur", "possrcs", "posrecs"} <= keys
    np.testing.assert_array_equal(pcur, ref)
