"""Two-step passes (time blocking, csrc/awc_tb.cuh) through the C ABI.

A depth-2 run applies the same arithmetic per node as depth-1 runs, so every
comparison here is exact (bitwise equal traces and fields); depth-1 runs are
themselves checked against the oracle in test_gpu_forward.py. Also: the
timeout path of the bounded pipeline waits, made to run out without a fault
(the producer withholds one plane load), and the context's recovery."""
import numpy as np
import pytest

import cases
from test_gpu_forward import CASES3D, small3d

pytestmark = pytest.mark.gpu

# every 3D case whose sources and receivers are interior nodes
TB_CASES = sorted(n for n in CASES3D if n != "rim_sources")


def _plan(pkg, ctx, case, precision):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    kw = dict(kw)
    kw.pop("check_ppw", None)
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    s = pkg.prepare(lengths, lt, vel, srcs, recs, precision=precision, ppw=1e-9, **kw)
    plan = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                    s["posrecs"])
    return s, plan


def _depth1(plan):
    plan.set_blocking(1)
    plan.reset()
    plan.run()
    return plan.traces(), plan.field()


@pytest.mark.parametrize("name", TB_CASES)
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_two_step_equals_one_step(pkg, ctx, name, precision):
    s, plan = _plan(pkg, ctx, CASES3D[name](), precision)
    try:
        ref_t, ref_p = _depth1(plan)
        assert np.abs(ref_t).max() > 0
        nt = s["nt"]
        for zchunks, rows in ((1, 16), (3, 8), (1000, 16), (2, 8)):
            plan.set_blocking(2, zchunks, rows)
            assert plan.get_blocking()[0] == 2 and plan.get_blocking()[2] == rows
            plan.reset()
            plan.run()
            np.testing.assert_array_equal(plan.traces(), ref_t)
            np.testing.assert_array_equal(plan.field(), ref_p)
        # eager launches, and a run split into odd pieces (one-step launches
        # in between)
        plan.reset()
        plan.run(graph=False)
        np.testing.assert_array_equal(plan.traces(), ref_t)
        plan.reset()
        plan.run(7)
        plan.run(nt // 3, graph=False)
        plan.run()
        assert plan.step == nt
        np.testing.assert_array_equal(plan.traces(), ref_t)
        np.testing.assert_array_equal(plan.field(), ref_p)
    finally:
        plan.close()


def test_depth_switches_mid_run(pkg, ctx):
    """The state carries over between depths: 5 one-step launches, then
    two-step passes, then one-step again, then two-step to the end."""
    s, plan = _plan(pkg, ctx, small3d(freetop=False), "f32")
    try:
        ref_t, ref_p = _depth1(plan)
        nt = s["nt"]
        plan.reset()
        plan.run(5)
        plan.set_blocking(2, 2)
        plan.run(nt // 2)
        plan.set_blocking(1)
        plan.run(3)
        plan.set_blocking(2, 1, 8)
        plan.run()
        assert plan.step == nt
        np.testing.assert_array_equal(plan.traces(), ref_t)
        np.testing.assert_array_equal(plan.field(), ref_p)
    finally:
        plan.close()


def test_launch_count(pkg, ctx):
    s, plan = _plan(pkg, ctx, CASES3D["core_and_bands"](), "f32")
    try:
        one = plan.launches_per_step
        assert plan.launch_count(11) == 11 * one
        plan.set_blocking(2, 2)
        # 5 passes of one or two launches (the tiles that meet an x or y band
        # and the others, when there are both), then one one-step launch
        n10 = plan.launch_count(10)
        assert n10 in (5, 10)
        assert plan.launch_count(11) == n10 + one
    finally:
        plan.close()


def test_rim_io_keeps_depth_one(pkg, ctx):
    """Sources or receivers on the Dirichlet rim need the three-buffer
    rotation of the reference; two-step passes are refused for them."""
    s, plan = _plan(pkg, ctx, CASES3D["rim_sources"](), "f32")
    try:
        with pytest.raises(pkg.AwcInvalidArgument, match="interior"):
            plan.set_blocking(2)
        assert plan.get_blocking()[0] == 1
    finally:
        plan.close()


def test_autotune_considers_depth_two(pkg, ctx):
    s, plan = _plan(pkg, ctx, CASES3D["core_and_bands"](), "f32")
    try:
        ref_t, ref_p = _depth1(plan)
        best = plan.autotune(6)
        assert best > 0 and plan.step == 0
        depth, zchunks, rows = plan.get_blocking()
        assert depth in (1, 2) and zchunks >= 1 and rows in (8, 16)
        plan.run()
        np.testing.assert_array_equal(plan.traces(), ref_t)
    finally:
        plan.close()


def test_bounded_wait_times_out_and_context_recovers(pkg, ctx, oracle):
    """The producer of every block withholds plane load 6, so each block's
    wait for that plane runs out after 4 tries of at most 2 us: the run
    returns AWC_ERR_TIMEOUT (the kernel drains its other loads and returns;
    nothing faults). With the default budget the next runs on the same
    context give the exact depth-1 results, and the traces match the
    oracle."""
    case = small3d(freetop=False)
    s, plan = _plan(pkg, ctx, case, "f64")
    try:
        ref_t, ref_p = _depth1(plan)
        plan.set_blocking(2, 1)
        plan.set_wait(rounds=4, round_ns=2000, withhold=6)
        plan.reset()
        with pytest.raises(pkg.AwcError) as ei:
            plan.run(4)
        assert ei.value.code == pkg._lib.AWC_ERR_TIMEOUT
        plan.set_wait()
        plan.reset()
        plan.run()
        np.testing.assert_array_equal(plan.traces(), ref_t)
        np.testing.assert_array_equal(plan.field(), ref_p)
    finally:
        plan.close()
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    so = oracle.setup(lengths, lt, vel, sp, t0s, f0, rp, **kw)
    _, tr_o = oracle.forward(so)
    assert cases.rel_l2(ref_t, tr_o) <= 1e-10
    # a fresh forward solve on the same context still works
    s2, plan2 = _plan(pkg, ctx, small3d(seed=3), "f32")
    try:
        plan2.run()
        assert np.all(np.isfinite(plan2.traces()))
    finally:
        plan2.close()
