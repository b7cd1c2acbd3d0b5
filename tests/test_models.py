"""Velocity-model input (models.py): rescalemod
(scripts/models/rescale_model.jl:19-55) and velocity_from_function
(src/shared/acoustic_3D_multixPU.jl:272-273). CPU only."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def M(pkg):
    from acousticwavecpml_b200 import models
    return models


def test_rescalemod_same_size_is_identity(M):
    rng = np.random.default_rng(0)
    a = rng.random((7, 5, 6))
    for kind in M.KINDS:
        np.testing.assert_allclose(M.rescalemod(7, 5, 6, kind, model=a), a, rtol=0, atol=1e-12)


def test_rescalemod_linear_is_exact_on_trilinear_data(M):
    i, j, k = np.meshgrid(np.arange(1, 9), np.arange(1, 7), np.arange(1, 6), indexing="ij")
    a = 2000.0 + 3.0 * i - 7.0 * j + 11.0 * k + 0.5 * i * j * k
    out = M.rescalemod(15, 11, 9, "linear", model=a)
    x, y, z = (np.linspace(1.0, n0, n) for n0, n in ((8, 15), (6, 11), (5, 9)))
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    np.testing.assert_allclose(out, 2000.0 + 3 * X - 7 * Y + 11 * Z + 0.5 * X * Y * Z,
                               rtol=1e-13)
    # the cubic spline is exact on data linear in each coordinate
    lin = 2000.0 + 3.0 * i - 7.0 * j + 11.0 * k
    np.testing.assert_allclose(M.rescalemod(15, 11, 9, "cubic", model=lin),
                               2000.0 + 3 * X - 7 * Y + 11 * Z, rtol=1e-12)


def test_rescalemod_nearest_rounds_like_julia(M):
    a = np.arange(4.0)[:, None, None] * np.ones((1, 1, 1))
    # LinRange(1, 4, 7) = 1, 1.5, 2, 2.5, 3, 3.5, 4: round(1.5) = 2, round(2.5) = 2,
    # round(3.5) = 4 (ties to even)
    out = M.rescalemod(7, 1, 1, "nearest", model=a)
    np.testing.assert_array_equal(out[:, 0, 0], [0.0, 1.0, 1.0, 1.0, 2.0, 3.0, 3.0])


def test_rescalemod_func_and_errors(M):
    rng = np.random.default_rng(3)
    a = rng.random((6, 6, 6))
    itp = M.rescalemod(0, 0, 0, "linear", model=a, func=True)
    assert itp(2, 3, 4) == pytest.approx(a[1, 2, 3])
    assert itp(2.5, 3, 4) == pytest.approx(0.5 * (a[1, 2, 3] + a[2, 2, 3]))
    with pytest.raises(ValueError):
        M.rescalemod(4, 4, 4, "spline7", model=a)
    with pytest.raises(ValueError):
        M.rescalemod(4, 4, 4, model=a[0])


def test_velocity_from_function(M):
    vel = M.velocity_from_function(lambda x, y, z: 1500.0 + 0.5 * y + 0.0 * x * z, (5, 4, 3),
                                   (10.0, 20.0, 30.0))
    assert vel.shape == (5, 4, 3) and vel.flags.f_contiguous
    np.testing.assert_allclose(vel[2, 3, 1], 1500.0 + 0.5 * 60.0)
    # a scalar-only function is evaluated node by node
    v2 = M.velocity_from_function(lambda x, y: 2000.0 if y < 15.0 else 2500.0, (3, 3),
                                  (10.0, 10.0))
    np.testing.assert_array_equal(v2[:, 1], 2000.0)
    np.testing.assert_array_equal(v2[:, 2], 2500.0)
    with pytest.raises(ValueError):
        M.velocity_from_function(lambda x, y: -1.0 + 0.0 * x, (3, 3), (1.0, 1.0))
