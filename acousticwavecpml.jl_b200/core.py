"""Host layer over the C ABI: contexts, device-resident plans and the solver
setup that solve2D/solve3D perform before their time loop.

`prepare()` restates the host part of solve2D/solve3D
(src/shared/acoustic_2D_xPU.jl:154-240, src/shared/acoustic_3D_xPU.jl:194-289):
grid spacing, CFL time step, step count, CPML coefficients (through the C
library), scaled source time functions and nearest-node snapping. Everything
after that runs on the GPU through libawcpml.so.
"""
import ctypes
import math
import threading

import numpy as np

from . import _lib
from ._lib import AWC_F32, AWC_F64, Problem, check

PRECISIONS = {"f32": AWC_F32, "float32": AWC_F32, "f64": AWC_F64, "float64": AWC_F64}


def _shape(p):
    """Array shape of a problem's fields: (nx,), (nx, ny) or (nx, ny, nz)."""
    return ((p.nx,), (p.nx, p.ny), (p.nx, p.ny, p.nz))[p.ndim - 1]


def _ptr(a):
    """Host address of a numpy array or a torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


class Context:
    """An awc_ctx on one device: stream, events and the plan/graph cache."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        check(_lib.lib().awc_create(ctypes.byref(self._h), int(device)))
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            _lib.lib().awc_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_run_ms(self):
        return float(_lib.lib().awc_last_run_ms(self._h))

    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return int(_lib.lib().awc_ctx_stream(self._h) or 0)

    def set_autotune(self, steps):
        """Steps per candidate of the launch-shape autotuning that forward()
        runs for each new 3D problem shape (0 disables it)."""
        check(_lib.lib().awc_ctx_set_autotune(self._h, int(steps)), self._h)

    def forward(self, problem, vel, coeffs, possrcs, dt2srctf, posrecs, traces, pfinal=None):
        """awc_forward on host buffers (numpy arrays or pinned torch tensors)."""
        rc = _lib.lib().awc_forward(self._h, ctypes.byref(problem), _ptr(vel), _ptr(coeffs),
                                    _ptr(possrcs), _ptr(dt2srctf), _ptr(posrecs), _ptr(traces),
                                    _ptr(pfinal))
        check(rc, self._h)

    def plan(self, problem, vel, coeffs, possrcs, dt2srctf, posrecs):
        return Plan(self, problem, vel, coeffs, possrcs, dt2srctf, posrecs)


_DEFAULT = {}
_LOCK = threading.Lock()


def forward_decomposed(contexts, problem, vel, coeffs, possrcs, dt2srctf, posrecs, traces,
                       pfinal=None):
    """awc_forward_decomposed: the shot split along its last axis into
    len(contexts) subdomains, subdomain s on contexts[s] (the same context
    may repeat), with a one-plane halo exchange per step."""
    hs = (ctypes.c_void_p * len(contexts))(*[c.handle.value for c in contexts])
    rc = _lib.lib().awc_forward_decomposed(hs, len(contexts), ctypes.byref(problem), _ptr(vel),
                                           _ptr(coeffs), _ptr(possrcs), _ptr(dt2srctf),
                                           _ptr(posrecs), _ptr(traces), _ptr(pfinal))
    check(rc, contexts[0].handle)


def default_context(device=0):
    """Per-device context shared by solve2D/solve3D calls of this process."""
    with _LOCK:
        c = _DEFAULT.get(device)
        if c is None:
            c = _DEFAULT[device] = Context(device)
        return c


class Plan:
    """Device-resident problem (awc_plan): inputs uploaded once, state in HBM."""

    def __init__(self, ctx, problem, vel, coeffs, possrcs, dt2srctf, posrecs):
        self.ctx = ctx
        self.problem = problem
        self._keep = (vel, coeffs, possrcs, dt2srctf, posrecs)
        self._h = ctypes.c_void_p()
        rc = _lib.lib().awc_plan_create(ctx.handle, ctypes.byref(problem), _ptr(vel),
                                        _ptr(coeffs), _ptr(possrcs), _ptr(dt2srctf),
                                        _ptr(posrecs), ctypes.byref(self._h))
        check(rc, ctx.handle)
        self._keep = None

    def close(self):
        if self._h:
            _lib.lib().awc_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        check(_lib.lib().awc_plan_reset(self._h), self.ctx.handle)

    def run(self, nsteps=None, graph=True):
        """Advances nsteps (default: to nt); returns the device time in ms."""
        if nsteps is None:
            nsteps = self.problem.nt
        ms = ctypes.c_float(0.0)
        check(_lib.lib().awc_plan_run(self._h, int(nsteps), 1 if graph else 0, ctypes.byref(ms)),
              self.ctx.handle)
        return float(ms.value)

    @property
    def step(self):
        return int(_lib.lib().awc_plan_step(self._h))

    @property
    def launches_per_step(self):
        return int(_lib.lib().awc_plan_launches_per_step(self._h))

    def set_launch(self, tile_y, zchunk, band_zchunk=10):
        """3D launch shape: core tile rows, core z chunk, band-kernel z chunk."""
        check(_lib.lib().awc_plan_set_launch(self._h, int(tile_y), int(zchunk),
                                             int(band_zchunk)), self.ctx.handle)

    def get_launch(self):
        ty, zc, bz = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(_lib.lib().awc_plan_get_launch(self._h, ctypes.byref(ty), ctypes.byref(zc),
                                             ctypes.byref(bz)), self.ctx.handle)
        return ty.value, zc.value, bz.value

    def set_blocking(self, depth, zchunks=2, rows=16):
        """Time steps per kernel pass (1 or 2), and the two-step kernel's z
        chunks per column tile and region rows (8 or 16); results do not
        depend on any of them."""
        check(_lib.lib().awc_plan_set_blocking(self._h, int(depth), int(rows), int(zchunks)),
              self.ctx.handle)

    def get_blocking(self):
        """(depth, zchunks, rows)."""
        d, r, z = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(_lib.lib().awc_plan_get_blocking(self._h, ctypes.byref(d), ctypes.byref(r),
                                               ctypes.byref(z)), self.ctx.handle)
        return d.value, z.value, r.value

    def launch_count(self, nsteps=None):
        """Kernel launches a run of nsteps (default: the remaining steps) issues."""
        if nsteps is None:
            nsteps = self.problem.nt
        return int(_lib.lib().awc_plan_launch_count(self._h, int(nsteps)))

    def run_snapshots(self, nsteps, nsave, out=None):
        """Advances nsteps and returns the fields after every step whose count
        since the reset is a multiple of nsave, as an array (k, *shape) of
        float64 (`out`, if given, must hold them: (max_snaps, *shape),
        C-contiguous over the snapshot index with column-major fields)."""
        p = self.problem
        shape = _shape(p)
        n = min(int(nsteps), p.nt - self.step)
        count = max(0, (self.step + n) // nsave - self.step // nsave)
        if out is None:
            out = np.zeros((max(count, 1),) + shape[::-1])
        got = ctypes.c_int64(0)
        check(_lib.lib().awc_plan_run_snapshots(self._h, int(nsteps), int(nsave), _ptr(out),
                                                int(out.shape[0]), ctypes.byref(got)),
              self.ctx.handle)
        # each snapshot is a column-major field: view it as (nx, ny[, nz])
        return [np.asfortranarray(out[j].T) for j in range(got.value)]

    def set_wait(self, rounds=4096, round_ns=1000000, withhold=-1):
        """Bounded-wait budget of the two-step kernel's pipeline; `withhold`
        (tests of the timeout path only) makes every block skip one load."""
        check(_lib.lib().awc_plan_set_wait(self._h, int(rounds), int(round_ns), int(withhold)),
              self.ctx.handle)

    def autotune(self, steps=20):
        """Picks the fastest launch shape on this plan's data; resets the state.
        Returns the best time per step in ms."""
        ms = ctypes.c_float(0.0)
        check(_lib.lib().awc_plan_autotune(self._h, int(steps), ctypes.byref(ms)),
              self.ctx.handle)
        return float(ms.value)

    def traces(self, out=None):
        p = self.problem
        if out is None:
            out = np.zeros((p.nt, p.nrec), order="F")
        check(_lib.lib().awc_plan_traces(self._h, _ptr(out)), self.ctx.handle)
        return out

    def field(self, out=None):
        p = self.problem
        shape = _shape(p)
        if out is None:
            out = np.zeros(shape, order="F")
        check(_lib.lib().awc_plan_field(self._h, _ptr(out)), self.ctx.handle)
        return out


def round_ties_up(x):
    """round(Int, x, RoundNearestTiesUp) for finite x (exact, no x + 0.5)."""
    x = np.asarray(x, dtype=np.float64)
    f = np.floor(x)
    return (f + ((x - f) >= 0.5)).astype(np.int64)


def eval_srctf(fn, times, t0, f0):
    """srctf.(times, t0, f0): vectorised call when the function allows it."""
    try:
        v = np.asarray(fn(times, t0, f0), dtype=np.float64)
        if v.shape == times.shape:
            return v
    except Exception:
        pass
    return np.array([fn(t, t0, f0) for t in times], dtype=np.float64)


def problem_coeffs(problem, rcoef, f0, vel_max):
    n = _lib.lib().awc_coeffs_len(ctypes.byref(problem))
    coeffs = np.zeros(max(int(n), 1))
    check(_lib.lib().awc_problem_coeffs(ctypes.byref(problem), float(rcoef), float(f0),
                                        float(vel_max), coeffs.ctypes.data_as(_lib._dp)))
    return coeffs


def prepare(lengths, lt, vel, srcs, recs, halo=20, rcoef=0.0001, ppw=10.0, freetop=True,
            precision="f64", dt=None, nt=None):
    """Host setup of solve1D/solve2D/solve3D. Returns a dict of the awc_forward
    inputs.

    dt/nt default to the reference's rule (dt = sqrt(ndim) / (vmax Σ 1/d_i) / 2,
    which is dx / vmax / 2 in 1D (acoustic_1D.jl); nt = ceil(lt/dt)); passing
    them fixes the step explicitly instead. 1D has no free top.
    """
    vel = np.asfortranarray(vel, dtype=np.float64)
    ndim = vel.ndim
    if ndim not in (1, 2, 3) or len(lengths) != ndim:
        raise ValueError("vel must be 1D, 2D or 3D and match the number of model lengths")
    if ndim == 1:
        freetop = False
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    shape = vel.shape
    f0 = srcs.freqdomain
    vel_max = float(vel.max())
    d = [float(lengths[a]) / (shape[a] - 1) for a in range(ndim)]
    if dt is None:
        dt = math.sqrt(ndim) / (vel_max * sum(1.0 / x for x in d)) / 2.0
    if nt is None:
        nt = int(math.ceil(lt / dt))
    assert math.sqrt(sum(x * x for x in d)) <= vel_max / (ppw * f0), \
        "Not enough points per wavelength!"
    times = np.arange(nt, dtype=np.float64) * dt
    scale = (dt * dt) / math.prod(d)
    dt2srctf = np.zeros((nt, srcs.n), order="F")
    for s in range(srcs.n):
        dt2srctf[:, s] = scale * eval_srctf(srcs.srctfs[s], times, srcs.t0s[s], f0)

    def snap(pos, what):
        pos = np.atleast_2d(np.asarray(pos, dtype=np.float64))
        if pos.shape[1] != ndim:
            raise ValueError(f"{what} positions need {ndim} columns")
        out = np.zeros(pos.shape, dtype=np.int64, order="F")
        for a in range(ndim):
            out[:, a] = round_ties_up(pos[:, a] / d[a] + 1.0)
        ok = all(np.all((out[:, a] >= 1) & (out[:, a] <= shape[a])) for a in range(ndim))
        assert ok, f"At least one {what} is not inside the model!"
        return out

    possrcs = snap(srcs.positions, "source")
    posrecs = snap(recs.positions, "receiver")
    problem = Problem(ndim=ndim, precision=PRECISIONS[precision], nx=shape[0],
                      ny=shape[1] if ndim >= 2 else 1, nz=shape[2] if ndim == 3 else 1,
                      halo=int(halo), freetop=1 if freetop else 0, dx=d[0],
                      dy=d[1] if ndim >= 2 else 1.0, dz=d[2] if ndim == 3 else 1.0,
                      dt=float(dt), nt=int(nt), nsrc=srcs.n, nrec=recs.n)
    coeffs = problem_coeffs(problem, rcoef, f0, vel_max)
    return dict(problem=problem, vel=vel, coeffs=coeffs, possrcs=possrcs, dt2srctf=dt2srctf,
                posrecs=posrecs, dt=float(dt), nt=int(nt), d=d, vel_max=vel_max, f0=f0)


def a_eff_words(problem):
    """The reference's effective-access word count per step
    (acoustic_3D_xPU.jl:520-528, acoustic_2D_xPU.jl:422-428)."""
    h = problem.halo
    nx, ny = problem.nx, problem.ny
    if problem.ndim == 1:  # acoustic_1D.jl's count
        return 2 * (4 * (h + 1) + (h + 1)) + 2 * (4 * (h + 1) + (h + 1)) + (4 * nx + nx)
    if problem.ndim == 2:
        return ((h + 1) * ny * 2 * 3 + (h + 1) * nx * 2 * 3 + (h + 1) * ny * 2 * 2 +
                (h + 1) * nx * 2 * 2 + 4 * nx * ny)
    nz = problem.nz
    return ((h + 1) * ny * nz * 2 * 3 + (h + 1) * nx * nz * 2 * 3 + (h + 1) * nx * ny * 2 * 3 +
            (h + 1) * ny * nz * 2 * 2 + (h + 1) * nx * nz * 2 * 2 + (h + 1) * nx * ny * 2 * 2 +
            4 * nx * ny * nz)


def alloc_words(problem):
    """The reference's allocated-memory word count (acoustic_3D_xPU.jl:512-518)."""
    h = problem.halo
    nx, ny = problem.nx, problem.ny
    if problem.ndim == 1:  # acoustic_1D.jl's count
        return 3 * nx + 2 * (h + 1) + 2 * h + 4 * (h + 1) + 4 * h
    if problem.ndim == 2:
        return (3 * nx * ny + 2 * (h + 1) * ny + 2 * h * ny + 2 * (h + 1) * nx + 2 * h * nx +
                4 * 2 * (h + 1) + 4 * 2 * h)
    nz = problem.nz
    return (3 * nx * ny * nz + 2 * (h + 1) * ny * nz + 2 * h * ny * nz + 2 * (h + 1) * nx * nz +
            2 * h * nx * nz + 2 * (h + 1) * nx * ny + 2 * h * nx * ny + 4 * 3 * (h + 1) +
            4 * 3 * h)


def word_bytes(problem):
    return 8 if problem.precision == AWC_F64 else 4
