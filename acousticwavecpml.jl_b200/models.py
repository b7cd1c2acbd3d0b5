"""Velocity-model input: resampling a gridded model and evaluating a velocity
function on the solver grid, the two ways the reference builds its models.

* ``rescalemod`` restates ``rescalemod`` (scripts/models/rescale_model.jl:19-55):
  a 3D model sampled at the points LinRange(1, n_orig, n) of every axis
  (1-based index coordinates) by B-spline interpolation of the chosen order.
  Orders "nearest" and "linear" are exact restatements of Interpolations.jl's
  BSpline(Constant()) and BSpline(Linear()). "quadratic" and "cubic" use an
  interpolating spline of that order through the samples, applied axis by
  axis ("cubic" with natural end conditions, "quadratic" with not-a-knot
  ones); the reference's Natural(OnCell()) end conditions place the spline's
  ends half a cell beyond the first and last samples, so these two orders
  agree with it inside the model and may differ within about a cell of its
  faces (this build cannot run Julia to pin them).
* ``velocity_from_function`` evaluates vel_func(x, y[, z]) at the node
  coordinates x = (i - 1) dx, ... (the model set-up of the multi-process
  solvers, src/shared/acoustic_3D_multixPU.jl:272-273, on one process).
"""
import math

import numpy as np

KINDS = ("nearest", "linear", "quadratic", "cubic")


def _nearest_index(x, n):
    """0-based sample of 1-based coordinate x: Julia's round (ties to even)."""
    return np.clip(np.round(x).astype(np.int64) - 1, 0, n - 1)


def _resample0(a, x, kind):
    """Values of `a` along its first axis at the 1-based coordinates x."""
    n = a.shape[0]
    if kind == "nearest":
        return a[_nearest_index(x, n)]
    if kind == "linear" or n <= (3 if kind == "cubic" else 2):
        f = np.clip(x - 1.0, 0.0, n - 1.0)
        i0 = np.minimum(np.floor(f).astype(np.int64), max(n - 2, 0))
        w = (f - i0).reshape((-1,) + (1,) * (a.ndim - 1))
        i1 = np.minimum(i0 + 1, n - 1)
        return (1.0 - w) * a[i0] + w * a[i1]
    from scipy.interpolate import make_interp_spline
    k = 3 if kind == "cubic" else 2
    spl = make_interp_spline(np.arange(1.0, n + 1.0), a, k=k,
                             bc_type="natural" if kind == "cubic" else None, axis=0)
    return spl(np.clip(x, 1.0, float(n)))


def _resample_axis(a, axis, x, kind):
    """Values of `a` along `axis` at the 1-based coordinates x."""
    return np.moveaxis(_resample0(np.moveaxis(a, axis, 0), x, kind), 0, axis)


def _read_model(flnamedset):
    path, dset = flnamedset
    try:
        import h5py
    except ImportError as e:
        raise RuntimeError("reading an HDF5 model needs h5py; pass the array as `model` "
                           "instead") from e
    with h5py.File(path, "r") as f:
        # HDF5.jl writes Julia's column-major arrays; h5py reads them with
        # the axes reversed
        return np.asarray(f[dset][()]).transpose()


def rescalemod(nx, ny, nz, kind="nearest", model=None, flnamedset=None, func=False):
    """Resample a 3D velocity model onto nx x ny x nz nodes.

    ``model`` is the original array (or read from ``flnamedset`` = (HDF5
    file, dataset), as the reference does); the new node (i, j, k) takes the
    model's value at the 1-based coordinates LinRange(1, n_orig, n)[i] per
    axis. With ``func=True`` a callable itp(x, y, z) of 1-based coordinates
    is returned instead. Returns a Fortran-ordered float64 array.
    """
    if kind not in KINDS:
        raise ValueError(f"kind must be one of {KINDS}")
    res = np.asarray(_read_model(flnamedset) if model is None else model, dtype=np.float64)
    if res.ndim != 3:
        raise ValueError("the model must be a 3D array")

    def evaluate(xs):
        out = res
        for axis, x in enumerate(xs):
            out = _resample_axis(out, axis, np.atleast_1d(np.asarray(x, dtype=np.float64)), kind)
        return out

    if func:
        def itp(x, y, z):
            v = evaluate((x, y, z))
            return v.item() if v.size == 1 else v
        return itp
    grids = [np.linspace(1.0, float(n0), int(n)) for n0, n in zip(res.shape, (nx, ny, nz))]
    return np.asfortranarray(evaluate(grids))


def velocity_from_function(vel_func, shape, spacing):
    """vel[i, j(, k)] = vel_func(x, y(, z)) at x = (i - 1) dx, y = (j - 1) dy,
    z = (k - 1) dz (1-based i, j, k), as solve3D_multi fills its model; the
    function is called on broadcast coordinate arrays when it accepts them,
    else node by node."""
    coords = np.meshgrid(*[np.arange(n, dtype=np.float64) * d for n, d in zip(shape, spacing)],
                         indexing="ij")
    try:
        vel = np.asarray(vel_func(*coords), dtype=np.float64)
        if vel.shape != tuple(shape):
            vel = np.broadcast_to(vel, tuple(shape))
    except (TypeError, ValueError):
        vel = np.empty(shape)
        for idx in np.ndindex(*shape):
            vel[idx] = vel_func(*(float(c[idx]) for c in coords))
    if not np.all(np.isfinite(vel)) or vel.min() <= 0.0 or math.isnan(float(vel.max())):
        raise ValueError("vel_func must give positive finite velocities")
    return np.asfortranarray(vel)
