"""Batched 2D shots: many sources over several velocity models of uneven size
advancing together on the GPU (awc_batch_* in include/awcpml.h).

Each shot is set up exactly as solve2D sets up a single shot
(src/shared/acoustic_2D_xPU.jl:154-240): the model's own grid spacing and
time step, CPML coefficients from the shot's source frequency, scaled source
time functions and snapped positions. All models share the number of steps.
The reference has no batched entry point; this is the multi-shot form of
solve2D.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import Problem, Shot, check
from .core import _ptr, default_context, prepare


class _Marshal:
    """ctypes views of a batch's inputs (models, velocity pointers, awc_shot
    array), keeping the numpy arrays they point into alive."""

    def __init__(self, models, vels, shot_setups, shot_models):
        self.models = (Problem * len(models))(*models)
        self.vels = [np.asfortranarray(v, dtype=np.float64) for v in vels]
        self.vptr = (ctypes.c_void_p * len(vels))(*[v.ctypes.data for v in self.vels])
        self.keep, shots = [], []
        for s, m in zip(shot_setups, shot_models):
            arrs = [np.ascontiguousarray(s["coeffs"], dtype=np.float64),
                    np.asfortranarray(s["possrcs"], dtype=np.int64),
                    np.asfortranarray(s["dt2srctf"], dtype=np.float64),
                    np.asfortranarray(s["posrecs"], dtype=np.int64)]
            self.keep.append(arrs)
            shots.append(Shot(model=int(m), nsrc=s["problem"].nsrc, nrec=s["problem"].nrec,
                              coeffs=arrs[0].ctypes.data, possrcs=arrs[1].ctypes.data,
                              dt2srctf=arrs[2].ctypes.data, posrecs=arrs[3].ctypes.data))
        self.shots = (Shot * len(shots))(*shots)
        self.nrec = [s["problem"].nrec for s in shot_setups]


class Batch:
    """A device-resident batch (awc_batch): models and shots uploaded once.

    models: one Problem per model (nsrc = nrec = 0; precision and nt common);
    vels: their velocity arrays; shot_setups: prepare() dicts, one per shot;
    shot_models: the model index of each shot."""

    def __init__(self, ctx, models, vels, shot_setups, shot_models):
        self.ctx = ctx
        a = _Marshal(models, vels, shot_setups, shot_models)
        self.models, self.shot_model, self.shot_nrec = a.models, list(shot_models), a.nrec
        self.nt = int(a.models[0].nt)
        self._h = ctypes.c_void_p()
        check(_lib.lib().awc_batch_create(ctx.handle, len(models), a.models, a.vptr,
                                          len(shot_setups), a.shots, ctypes.byref(self._h)),
              ctx.handle)

    @property
    def nshots(self):
        return len(self.shot_nrec)

    def close(self):
        if self._h:
            _lib.lib().awc_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        check(_lib.lib().awc_batch_reset(self._h), self.ctx.handle)

    def run(self, nsteps=None, graph=True):
        ms = ctypes.c_float(0.0)
        n = self.nt if nsteps is None else nsteps
        check(_lib.lib().awc_batch_run(self._h, int(n), 1 if graph else 0, ctypes.byref(ms)),
              self.ctx.handle)
        return float(ms.value)

    @property
    def step(self):
        return int(_lib.lib().awc_batch_step(self._h))

    def set_launch(self, tile_y, blocks_per_sm):
        check(_lib.lib().awc_batch_set_launch(self._h, int(tile_y), int(blocks_per_sm)),
              self.ctx.handle)

    def get_launch(self):
        a, b = ctypes.c_int32(), ctypes.c_int32()
        check(_lib.lib().awc_batch_get_launch(self._h, ctypes.byref(a), ctypes.byref(b)),
              self.ctx.handle)
        return a.value, b.value

    def autotune(self, steps=20):
        ms = ctypes.c_float(0.0)
        check(_lib.lib().awc_batch_autotune(self._h, int(steps), ctypes.byref(ms)),
              self.ctx.handle)
        return float(ms.value)

    def traces(self, shot, out=None):
        if out is None:
            out = np.zeros((self.nt, self.shot_nrec[shot]), order="F")
        check(_lib.lib().awc_batch_traces(self._h, int(shot), _ptr(out)), self.ctx.handle)
        return out

    def field(self, shot):
        p = self.models[self.shot_model[shot]]
        out = np.zeros((p.nx, p.ny), order="F")
        check(_lib.lib().awc_batch_field(self._h, int(shot), _ptr(out)), self.ctx.handle)
        return out


def forward_batch(ctx, models, vels, shot_setups, shot_models):
    """awc_forward_batch: one call that uploads, autotunes (nt >= 100), runs
    every shot for nt steps and returns the traces (nt x nrec) per shot."""
    a = _Marshal(models, vels, shot_setups, shot_models)
    outs = [np.zeros((int(a.models[0].nt), n), order="F") for n in a.nrec]
    optr = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    check(_lib.lib().awc_forward_batch(ctx.handle, len(models), a.models, a.vptr,
                                       len(shot_setups), a.shots, optr), ctx.handle)
    return outs


def prepare_batch(models, shots, *, nt, halo=20, rcoef=0.0001, ppw=10.0, freetop=True,
                  precision="f32", dt=None):
    """models: list of (lx, ly, vel); shots: list of (model index, Sources,
    Receivers). Returns (Problem per used model, its vel, prepare() dict per
    shot, batch model index per shot). dt defaults to each model's own CFL
    step; nt is common to all models. Models that no shot uses are dropped."""
    setups = []
    for m, srcs, recs in shots:
        lx, ly, vel = models[m]
        setups.append(prepare((lx, ly), None, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw,
                              freetop=freetop, precision=precision, dt=dt, nt=nt))
    used = sorted({m for m, _, _ in shots})
    remap = {m: k for k, m in enumerate(used)}
    idx = [remap[m] for m, _, _ in shots]
    probs, vels = [], []
    for m in used:
        p = setups[idx.index(remap[m])]["problem"]
        probs.append(Problem(ndim=2, precision=p.precision, nx=p.nx, ny=p.ny, nz=1,
                             halo=p.halo, freetop=p.freetop, dx=p.dx, dy=p.dy, dz=1.0,
                             dt=p.dt, nt=p.nt, nsrc=0, nrec=0))
        vels.append(np.asfortranarray(models[m][2], dtype=np.float64))
    return probs, vels, setups, idx


def solve2D_batch(models, shots, *, nt, halo=20, rcoef=0.0001, ppw=10.0, freetop=True,
                  precision="f32", dt=None, device=0, autotune=20):
    """Runs every shot (model index, Sources, Receivers) over its model
    (lx, ly, vel) for nt steps in one batch and fills each shot's
    Receivers.seismograms (nt x nrec), like solve2D does for one shot."""
    probs, vels, setups, idx = prepare_batch(models, shots, nt=nt, halo=halo, rcoef=rcoef,
                                             ppw=ppw, freetop=freetop, precision=precision,
                                             dt=dt)
    ctx = default_context(device)
    b = Batch(ctx, probs, vels, setups, idx)
    try:
        if autotune and nt >= 100:
            b.autotune(autotune)
        b.run()
        for k, (_, _, recs) in enumerate(shots):
            recs.seismograms = b.traces(k)
    finally:
        b.close()
    return [recs.seismograms for _, _, recs in shots]


def shard(items, rank, world):
    """The items rank `rank` of `world` takes: rank, rank + world, ... (shots
    are independent, so a shot set splits over ranks with no exchange)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    return list(items)[rank::world]


def solve_sharded(shots, run_shots, group=None):
    """Runs a shot set over the ranks of a torch.distributed group: each rank
    calls run_shots(its shard) -> one result per shot (a traces array, say),
    and every rank gets all results back in the order of `shots` (one
    all_gather of the per-rank lists). Without an initialised process group
    it runs every shot locally."""
    import torch.distributed as dist

    on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if on else 0
    world = dist.get_world_size(group) if on else 1
    mine = run_shots(shard(shots, rank, world))
    if len(mine) != len(shard(shots, rank, world)):
        raise ValueError("run_shots must return one result per shot")
    if not on:
        return list(mine)
    parts = [None] * world
    dist.all_gather_object(parts, list(mine), group=group)
    out = [None] * len(shots)
    for r in range(world):
        out[r::world] = parts[r]
    return out


def solve2D_batch_sharded(models, shots, *, nt, group=None, **kw):
    """solve2D_batch over the ranks of a torch.distributed group (one GPU per
    rank, the device of the current CUDA context): rank r batches shots
    r, r + N, ... and every rank's Receivers get all seismograms."""
    traces = solve_sharded(shots, lambda mine: solve2D_batch(models, mine, nt=nt, **kw) if mine
                           else [], group)
    for (_, _, recs), tr in zip(shots, traces):
        recs.seismograms = tr
    return traces
