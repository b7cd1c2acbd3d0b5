"""Gradients of a trace misfit with respect to c² (the squared velocity), by
the discrete adjoint of the CPML time step (awc_misfit_gradient and
awc_adjoint_sources in include/awcpml.h).

The reference has no gradient. These functions take the same shot set-up as
solve2D/solve3D (a prepare() dict) and add:
  * misfit_gradient: J = 1/2 Σ (traces - observed)² and dJ/d(c²), with the
    forward state checkpointed every k steps and recomputed per segment;
  * misfit_gradient_shots: the same summed over the shots of one model in
    one call (the model uploaded once, the gradients summed on the device);
  * adjoint_sources: the transpose of the map from injected source values to
    traces, for dot-product tests;
  * C2Misfit: a torch.autograd.Function over c², so the solver takes part in
    a torch optimisation loop (the Python counterpart of a ChainRulesCore
    rrule);
  * sharded_gradient: the sum over shots of misfits and gradients when the
    shots are spread over the ranks of a torch.distributed group, with one
    all-reduce of the gradient and the misfit.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check
from .core import _ptr, default_context, prepare


def misfit_gradient(s, observed, checkpoint_every=50, ctx=None):
    """(J, dJ/dc² with vel's shape, traces (nt x nrec)) of the shot set up in
    `s` (prepare()) against `observed` (nt x nrec)."""
    ctx = ctx or default_context()
    p = s["problem"]
    obs = np.asfortranarray(observed, dtype=np.float64)
    if obs.shape != (p.nt, p.nrec):
        raise ValueError(f"observed must be (nt, nrec) = ({p.nt}, {p.nrec})")
    grad = np.zeros(s["vel"].shape, order="F")
    traces = np.zeros((p.nt, p.nrec), order="F")
    J = ctypes.c_double(0.0)
    check(_lib.lib().awc_misfit_gradient(ctx.handle, ctypes.byref(p), _ptr(s["vel"]),
                                         _ptr(s["coeffs"]), _ptr(s["possrcs"]),
                                         _ptr(s["dt2srctf"]), _ptr(s["posrecs"]), _ptr(obs),
                                         int(checkpoint_every), ctypes.byref(J), _ptr(grad),
                                         _ptr(traces)), ctx.handle)
    return float(J.value), grad, traces


def stack_shots(setups, observed):
    """The stacked inputs of awc_misfit_gradient_shots, checked: (possrcs
    (nsrc, ndim, nshot) int64, dt2srctf (nt, nsrc, nshot), observed (nt,
    nrec, nshot)), Fortran-ordered, so that shot s's block starts at
    s * nsrc * ndim, s * nt * nsrc and s * nt * nrec. Raises ValueError when
    the shots do not share the problem, vel, coeffs and receivers."""
    if not setups:
        raise ValueError("no shots")
    s0 = setups[0]
    p = s0["problem"]

    def same(a, b):
        return a is b or np.array_equal(a, b)

    for s in setups[1:]:
        q = s["problem"]
        if any(getattr(q, f) != getattr(p, f) for f, _ in type(p)._fields_):
            raise ValueError("every shot needs the same problem (grid, nt, nsrc, nrec)")
        if not (same(s["vel"], s0["vel"]) and same(s["coeffs"], s0["coeffs"])
                and same(s["posrecs"], s0["posrecs"])):
            raise ValueError("every shot needs the same vel, coeffs and receivers")
    if isinstance(observed, np.ndarray) and observed.ndim == 3:
        obs = np.asfortranarray(observed, dtype=np.float64)
    else:
        if len(observed) != len(setups):
            raise ValueError("one observed array per shot")
        obs = np.stack([np.asarray(o, dtype=np.float64) for o in observed], axis=-1)
        obs = np.asfortranarray(obs)
    if obs.shape != (p.nt, p.nrec, len(setups)):
        raise ValueError(f"observed must be (nt, nrec) = ({p.nt}, {p.nrec}) per shot")
    pos = np.asfortranarray(np.stack([np.asarray(s["possrcs"], dtype=np.int64) for s in setups],
                                     axis=-1))
    stf = np.asfortranarray(np.stack([np.asarray(s["dt2srctf"], dtype=np.float64)
                                      for s in setups], axis=-1))
    return pos, stf, obs


def misfit_gradient_shots(setups, observed, checkpoint_every=50, ctx=None):
    """(Σ J, Σ dJ/dc²) over shots of one model, equal to summing
    misfit_gradient over the shots in order. setups[s] is shot s's prepare()
    dict: all share the problem, vel, coeffs and receivers, and only their
    sources differ. observed: one (nt x nrec) array per shot, or all of them
    as one (nt x nrec x nshot) array (used without a copy when it is a
    Fortran-ordered float64 array)."""
    pos, stf, obs = stack_shots(setups, observed)
    ctx = ctx or default_context()
    s0 = setups[0]
    p = s0["problem"]
    grad = np.zeros(s0["vel"].shape, order="F")
    J = ctypes.c_double(0.0)
    check(_lib.lib().awc_misfit_gradient_shots(ctx.handle, ctypes.byref(p), len(setups),
                                               _ptr(s0["vel"]), _ptr(s0["coeffs"]), _ptr(pos),
                                               _ptr(stf), _ptr(s0["posrecs"]), _ptr(obs),
                                               int(checkpoint_every), ctypes.byref(J),
                                               _ptr(grad)), ctx.handle)
    return float(J.value), grad


def adjoint_sources(s, adjoint_traces, ctx=None):
    """Aᵀ r: the adjoint of the injected source values (nt x nsrc) for the
    adjoint traces r (nt x nrec), with c fixed as in `s`."""
    ctx = ctx or default_context()
    p = s["problem"]
    r = np.asfortranarray(adjoint_traces, dtype=np.float64)
    if r.shape != (p.nt, p.nrec):
        raise ValueError(f"adjoint_traces must be (nt, nrec) = ({p.nt}, {p.nrec})")
    out = np.zeros((p.nt, p.nsrc), order="F")
    check(_lib.lib().awc_adjoint_sources(ctx.handle, ctypes.byref(p), _ptr(s["vel"]),
                                         _ptr(s["coeffs"]), _ptr(s["possrcs"]),
                                         _ptr(s["posrecs"]), _ptr(r), _ptr(out)), ctx.handle)
    return out


def _with_c2(s, c2):
    """A copy of set-up `s` whose velocity is sqrt(c2); dt, coefficients and
    sources stay as they are."""
    t = dict(s)
    t["vel"] = np.asfortranarray(np.sqrt(np.asarray(c2, dtype=np.float64)))
    return t


def gradient(lengths, lt, vel, srcs, recs, observed, *, halo=20, rcoef=0.0001, ppw=10.0,
             freetop=True, precision="f64", dt=None, nt=None, checkpoint_every=50, device=0):
    """Misfit and dJ/d(c²) of one shot, set up like solve2D/solve3D (same
    arguments); fills recs.seismograms with the modelled traces."""
    s = prepare(lengths, lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw, freetop=freetop,
                precision=precision, dt=dt, nt=nt)
    J, grad, traces = misfit_gradient(s, observed, checkpoint_every, default_context(device))
    recs.seismograms = traces
    return J, grad


try:
    import torch

    class C2Misfit(torch.autograd.Function):
        """J(c²) for a fixed shot set-up; backward returns dJ/dc² (float64
        CPU tensors). Usage: J = C2Misfit.apply(c2, s, observed, k)."""

        @staticmethod
        def forward(fctx, c2, s, observed, checkpoint_every=50):
            J, grad, _ = misfit_gradient(_with_c2(s, c2.detach().cpu().numpy()), observed,
                                         checkpoint_every)
            fctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(grad)).reshape(c2.shape))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(fctx, gJ):
            (grad,) = fctx.saved_tensors
            return gJ * grad.to(gJ.device), None, None, None
except ImportError:  # torch is optional for the C-ABI users of this package
    C2Misfit = None


def sharded_gradient(shots, shot_gradient, shape, group=None, batched=False):
    """Σ over shots of (J, dJ/dc²) when each rank of a torch.distributed group
    takes shots rank, rank + N, ...: every rank calls shot_gradient(shot) ->
    (J, grad ndarray of `shape`) for its share, sums them, and one all-reduce
    (sum) of [grad, J] gives every rank the total. With batched=True the rank
    makes one call, shot_gradient(list of its shots) -> their summed (J, grad)
    (e.g. misfit_gradient_shots). Without an initialised process group it sums
    all shots locally."""
    import torch
    import torch.distributed as dist

    on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if on else 0
    world = dist.get_world_size(group) if on else 1
    total = np.zeros(shape, order="F")  # the layout misfit_gradient returns
    tt = torch.from_numpy(total.reshape(-1, order="F"))  # a view: torch adds on all cores
    J = 0.0
    mine = list(shots[rank::world])
    calls = ([mine] if mine else []) if batched else mine
    for shot in calls:
        j, g = shot_gradient(shot)
        J += j
        g = np.asarray(g, dtype=np.float64)
        if g.shape != total.shape:
            raise ValueError(f"shot_gradient returned shape {g.shape}, expected {total.shape}")
        gv = g if g.flags.f_contiguous else np.asfortranarray(g)
        tt.add_(torch.from_numpy(gv.reshape(-1, order="F")))
    if on:
        buf = torch.from_numpy(np.concatenate([total.ravel(order="F"), [J]]))
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        buf = buf.to(dev)
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        buf = buf.cpu().numpy()
        J = float(buf[-1])
        total = buf[:-1].reshape(total.shape, order="F")
    return J, total
