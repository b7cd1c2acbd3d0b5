"""Host-side logic of the library and its Python mirror (CPU only: no call
here launches a kernel)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "awcpml.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(awc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._lib.lib()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    # and the ctypes table covers the header exactly
    assert sorted(pkg._lib.SIGNATURES) == names


@pytest.mark.parametrize("halo", [0, 1, 5, 20])
@pytest.mark.parametrize("onwhere", ["ongrd", "halfgrd"])
def test_cpml_coeffs_match_oracle_bitwise(pkg, oracle, halo, onwhere):
    args = (halo, 1.7677669529663688e-3, 2.0, 1381.55, math.pi * 10.0, 1.0, onwhere)
    got = pkg.calc_Kab_CPML(*args)
    ref = oracle.calc_Kab_CPML(*args)
    for g, r in zip(got, ref):
        assert g.shape == r.shape == (halo + (onwhere == "halfgrd"),)
        np.testing.assert_array_equal(g, r)


def test_calc_Kab_CPML_rejects_bad_onwhere(pkg):
    with pytest.raises(ValueError):
        pkg.calc_Kab_CPML(20, 1e-3, 2.0, 1.0, 1.0, 1.0, "nowhere")


def test_cpml_profile_shape(pkg):
    # left side decays toward the interior, right side mirrors it; staggered
    # profile starts with distance 0 (utils.jl:35-38)
    a_l, a_r, bK_l, bK_r = pkg.calc_Kab_CPML(20, 1e-3, 2.0, 2000.0, math.pi * 10, 1.0, "ongrd")
    np.testing.assert_allclose(a_l, a_r[::-1], rtol=0, atol=0)
    assert a_l[0] < a_l[-1] < 0 or a_l[-1] == 0.0
    assert np.all(bK_l <= 1.0) and np.all(bK_l > 0.0)


@pytest.mark.parametrize("case", [lambda: cases.ref_center(True), cases.ref_gradient])
def test_prepare_matches_oracle_setup(pkg, oracle, case):
    lengths, lt, vel, sp, t0s, f0, rp, kw = case()
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D] * len(t0s), f0)
    recs = pkg.Receivers(rp)
    s = pkg.prepare(lengths, lt, vel, srcs, recs, **kw)
    o = oracle.setup(lengths, lt, vel, sp, t0s, f0, rp, **kw)
    assert s["dt"] == o["dt"] and s["nt"] == o["nt"]
    np.testing.assert_array_equal(s["possrcs"], o["possrcs"])
    np.testing.assert_array_equal(s["posrecs"], o["posrecs"])
    np.testing.assert_array_equal(s["coeffs"], o["coeffs"])
    np.testing.assert_array_equal(s["dt2srctf"], o["dt2srctf"])


def test_prepare_explicit_dt_nt(pkg):
    from acousticwavecpml_b200 import workloads as W
    w = W.config1()
    srcs, recs = W.sources_receivers(pkg, w)
    s = pkg.prepare(w["lengths"], w["lt"], w["vel"], srcs, recs, **w["kwargs"])
    p = s["problem"]
    assert (p.nx, p.ny, p.nt, p.nrec) == (241, 241, 1000, 21)
    assert s["possrcs"].tolist() == [[121, 121]]
    assert s["posrecs"][:, 1].tolist() == [31] * 21
    assert s["posrecs"][:, 0].tolist() == list(range(21, 222, 10))
    assert p.dt == 0.7 * 10.0 / (2000.0 * math.sqrt(2.0))


def test_round_ties_up(pkg):
    from acousticwavecpml_b200.core import round_ties_up
    x = np.array([0.5, 1.5, 2.5, -0.5, -1.5, 0.49999999999999994, 2.4999999999999996, 3.0])
    assert round_ties_up(x).tolist() == [1, 2, 3, 0, -1, 0, 2, 3]


def test_sources_receivers_assertions(pkg):
    with pytest.raises(AssertionError):
        pkg.Sources(np.zeros((0, 2)), [], [], 10.0)
    with pytest.raises(AssertionError):
        pkg.Sources([[1.0, 1.0]], [0.1, 0.2], [pkg.rickersource1D], 10.0)
    with pytest.raises(AssertionError):
        pkg.Receivers(np.zeros((0, 3)))


def test_prepare_errors_like_reference(pkg):
    lengths, lt, vel, sp, t0s, f0, rp, kw = cases.ref_center(False)
    srcs = pkg.Sources(sp, t0s, [pkg.rickersource1D], f0)
    bad = pkg.Receivers([[5000.0, 10.0]])
    with pytest.raises(AssertionError, match="not inside the model"):
        pkg.prepare(lengths, lt, vel, srcs, bad, **kw)
    recs = pkg.Receivers(rp)
    with pytest.raises(AssertionError, match="points per wavelength"):
        pkg.prepare(lengths, lt, vel, pkg.Sources(sp, t0s, [pkg.rickersource1D], 1000.0), recs,
                    **kw)


def _problem(pkg, **over):
    d = dict(ndim=3, precision=pkg.AWC_F32, nx=40, ny=30, nz=20, halo=5, freetop=1, dx=10.0,
             dy=10.0, dz=10.0, dt=1e-3, nt=10, nsrc=1, nrec=1)
    d.update(over)
    return pkg.Problem(**d)


@pytest.mark.parametrize("over", [
    dict(ndim=4), dict(precision=7), dict(nx=2), dict(halo=-1), dict(halo=19),
    dict(dt=0.0), dict(dx=-1.0), dict(nt=-1), dict(ndim=2, nz=5)])
def test_problem_validation(pkg, over):
    p = _problem(pkg, **over)
    coeffs = np.zeros(1000)
    rc = pkg._lib.lib().awc_problem_coeffs(ctypes.byref(p), 1e-4, 10.0, 2000.0,
                                           coeffs.ctypes.data_as(pkg._lib._dp))
    assert rc == pkg._lib.AWC_ERR_INVALID
    assert pkg._lib.lib().awc_last_error(None)


def test_coeffs_len(pkg):
    p = _problem(pkg, halo=20)
    assert pkg._lib.lib().awc_coeffs_len(ctypes.byref(p)) == 3 * (8 * 20 + 4)
    p = _problem(pkg, ndim=2, nz=1, halo=0)
    assert pkg._lib.lib().awc_coeffs_len(ctypes.byref(p)) == 2 * 4


def test_ricker_matches_reference_formula(pkg):
    t = np.linspace(0, 1, 101)
    out = np.zeros_like(t)
    rc = pkg._lib.lib().awc_ricker(t.size, t.ctypes.data_as(pkg._lib._dp), 0.4, 10.0,
                                   out.ctypes.data_as(pkg._lib._dp))
    assert rc == 0
    x = math.pi * 10.0 * (t - 0.4)
    np.testing.assert_allclose(out, (1 - 2 * x * x) * np.exp(-x * x), rtol=1e-15, atol=1e-300)
    np.testing.assert_allclose(pkg.rickersource1D(t, 0.4, 10.0), out, rtol=1e-15, atol=1e-300)


def test_a_eff_matches_reference_formula(pkg):
    from acousticwavecpml_b200.core import a_eff_words
    p = _problem(pkg, nx=296, ny=276, nz=296, halo=20)
    h, nx, ny, nz = 20, 296, 276, 296
    ref = ((h + 1) * ny * nz * 2 * 3 + (h + 1) * nx * nz * 2 * 3 + (h + 1) * nx * ny * 2 * 3 +
           (h + 1) * ny * nz * 2 * 2 + (h + 1) * nx * nz * 2 * 2 + (h + 1) * nx * ny * 2 * 2 +
           4 * nx * ny * nz)
    assert a_eff_words(p) == ref
    assert abs(ref * 4 / 1e6 - 597.8) < 0.1  # MB per step in FP32


def test_bench_min_traffic(pkg):
    """The bench line's minimal traffic at 296 x 276 x 296 (halo 20, free
    top): 4 field words per interior node plus a read and a write of every
    live ψ (h + 1 layers) and ξ (h layers) entry, FP32."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    p = _problem(pkg, nx=296, ny=276, nz=296, halo=20, freetop=1)
    cells = 294 * 274 * 294
    band = 2 * 2 * 41 * (274 * 294) + 1 * 2 * 41 * (294 * 294) + 2 * 2 * 41 * (294 * 274)
    assert bench.min_traffic(p) == 4 * (4 * cells + band) == 512975904
    p.freetop = 0
    band += 2 * 41 * (294 * 294)
    assert bench.min_traffic(p) == 4 * (4 * cells + band)


def test_create_without_device_fails_cleanly(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.AwcError) as e:
        pkg.Context(0)
    assert e.value.code == pkg._lib.AWC_ERR_NODEVICE
