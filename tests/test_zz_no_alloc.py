"""awc_forward2d_f32_static: the 2D FP32 forward solve for callers that
cannot let the library allocate device memory (a loop that must not stall on
cudaMalloc's device synchronisation, or a framework whose allocator owns all
device memory). It keeps its state in one fixed device array. These tests
call it through the C ABI and compare it with awc_forward.

This file is collected last so that a failure here comes after every other
test has run."""
import ctypes

import numpy as np
import pytest

import cases


def _setup(pkg, case, precision="f32"):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    return pkg.prepare(lengths, lt, vel, srcs, recs, precision=precision, **kw)


def _static(pkg, s):
    p = s["problem"]
    traces = np.zeros((p.nt, p.nrec), order="F")
    pend = np.zeros(s["vel"].shape, order="F")
    rc = pkg._lib.lib().awc_forward2d_f32_static(
        ctypes.byref(p), s["vel"].ctypes.data, s["coeffs"].ctypes.data, s["possrcs"].ctypes.data,
        s["dt2srctf"].ctypes.data, s["posrecs"].ctypes.data, traces.ctypes.data, pend.ctypes.data)
    return rc, traces, pend


@pytest.mark.gpu
def test_static_matches_awc_forward_twice(pkg):
    """Two calls in a row, each equal to awc_forward within the FP32 tolerance
    of the other tests (1e-4 relative L2), traces and final field. The runs
    stop while the wavefield is still inside the model: after it has left, the
    final field is a residual ~1e-5 of its peak, on which any FP32 rounding
    difference shows up as a large relative error. The second call starts
    from the first one's leftover array contents."""
    ctx = pkg.default_context(0)
    for case, nt in ((cases.ref_gradient(), 700), (cases.ref_center(False), 400)):
        case = case[:7] + (dict(case[7], nt=nt),)
        s = _setup(pkg, case)
        p = s["problem"]
        tr_ref = np.zeros((p.nt, p.nrec), order="F")
        pe_ref = np.zeros(s["vel"].shape, order="F")
        ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr_ref,
                    pe_ref)
        assert np.abs(tr_ref).max() > 0 and np.abs(pe_ref).max() > 0
        for _ in range(2):
            rc, tr, pe = _static(pkg, s)
            assert rc == 0, pkg._lib.lib().awc_last_error(None)
            assert cases.rel_l2(tr, tr_ref) <= 1e-4
            assert cases.rel_l2(pe, pe_ref) <= 1e-4


def test_static_rejects_oversized_and_unsupported_problems(pkg):
    """Checked before any device work, so this runs without a GPU too."""
    from acousticwavecpml_b200 import workloads as W
    w = W.config1()
    srcs, recs = W.sources_receivers(pkg, w)
    big = dict(w)
    big["vel"] = np.full((2000, 2000), 2000.0, order="F")  # 4M nodes > 32 MiB of state
    s = pkg.prepare((19990.0, 19990.0), None, big["vel"], srcs, recs, precision="f32",
                    **w["kwargs"])
    rc, _, _ = _static(pkg, s)
    assert rc == pkg._lib.AWC_ERR_INVALID
    assert b"bytes of device scratch" in pkg._lib.lib().awc_last_error(None)
    s64 = pkg.prepare(w["lengths"], w["lt"], w["vel"], srcs, recs, precision="f64",
                      **w["kwargs"])
    rc, _, _ = _static(pkg, s64)
    assert rc == pkg._lib.AWC_ERR_INVALID


def test_static_rejects_bad_scalars_before_any_device_work(pkg):
    """nt beyond 2^31 (whose trace and source sizes would wrap a 64-bit byte
    count near 2^41), non-finite spacing or dt, and NULL arrays are refused on
    the host with AWC_ERR_INVALID, the limits awc_forward applies; no device
    memory is touched, so this runs without a GPU."""
    from acousticwavecpml_b200 import workloads as W
    w = W.config1()
    srcs, recs = W.sources_receivers(pkg, w)
    s = pkg.prepare(w["lengths"], w["lt"], w["vel"], srcs, recs, precision="f32", **w["kwargs"])
    p = s["problem"]
    lib = pkg._lib.lib()
    for field, value in (("nt", (1 << 41) + 3), ("nt", (1 << 31) + 1), ("nt", -1),
                         ("dx", float("inf")), ("dy", float("nan")), ("dt", float("inf")),
                         ("dt", 0.0)):
        bad = pkg._lib.Problem.from_buffer_copy(p)
        setattr(bad, field, value)
        rc = lib.awc_forward2d_f32_static(
            ctypes.byref(bad), s["vel"].ctypes.data, s["coeffs"].ctypes.data,
            s["possrcs"].ctypes.data, s["dt2srctf"].ctypes.data, s["posrecs"].ctypes.data,
            None, None)
        assert rc == pkg._lib.AWC_ERR_INVALID, (field, value)
        msg = lib.awc_last_error(None)
        assert (b"nt out of range" in msg) if field == "nt" else (b"positive and finite" in msg)
    rc = lib.awc_forward2d_f32_static(ctypes.byref(p), None, s["coeffs"].ctypes.data,
                                      s["possrcs"].ctypes.data, s["dt2srctf"].ctypes.data,
                                      s["posrecs"].ctypes.data, None, None)
    assert rc == pkg._lib.AWC_ERR_INVALID
    assert b"NULL" in lib.awc_last_error(None)
