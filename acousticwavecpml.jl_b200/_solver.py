"""Shared body of solve2D/solve3D: setup, one awc_forward call (or a plan run
with snapshots), outputs."""
import os

import numpy as np

from .core import _shape, a_eff_words, alloc_words, default_context, prepare, word_bytes


def _size_str(problem):
    if problem.ndim == 1:
        return f"{problem.nx}"
    if problem.ndim == 2:
        return f"{problem.nx}x{problem.ny}"
    return f"{problem.nx}x{problem.ny}x{problem.nz}"


def _write_snapshot(path, lengths, halo, pcur, possrcs, posrecs):
    """One snapshot file with the datasets of the reference's HDF5 files
    (acoustic_3D_xPU.jl:479-498): lx, ly, lz, halo, pcur, possrcs, posrecs.
    HDF5 (.h5) when h5py is importable, else numpy's .npz with the same
    names."""
    data = dict(lx=float(lengths[0]), halo=int(halo), pcur=pcur, possrcs=possrcs,
                posrecs=posrecs)
    for name, a in (("ly", 1), ("lz", 2)):
        if len(lengths) > a:
            data[name] = float(lengths[a])
    try:
        import h5py
    except ImportError:
        h5py = None
    if h5py is not None:
        path = path + ".h5"
        if os.path.exists(path):
            os.remove(path)
        with h5py.File(path, "w") as f:
            for k, v in data.items():
                f[k] = v
    else:
        path = path + ".npz"
        np.savez(path, **data)
    return path


def _run_with_snapshots(ctx, s, lengths, halo, nsave, save_name, save_dir, chunk_snaps=8):
    """The time loop of `s` with a snapshot after every step it (1-based) with
    it % nsave == 0, each written to save_dir/{save_name}_it{it} as it comes
    (the do_save branch of solve3D). Returns (traces, final field, files)."""
    p = s["problem"]
    os.makedirs(save_dir, exist_ok=True)
    plan = ctx.plan(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"])
    files = []
    try:
        if p.ndim == 3 and p.nt >= 100:
            plan.autotune(10)
        buf = np.zeros((chunk_snaps,) + _shape(p)[::-1])
        while plan.step < p.nt:
            start = plan.step
            snaps = plan.run_snapshots(nsave * chunk_snaps - start % nsave, nsave, buf)
            first_it = (start // nsave + 1) * nsave
            for j, field in enumerate(snaps):
                it = first_it + j * nsave
                files.append(_write_snapshot(os.path.join(save_dir, f"{save_name}_it{it}"),
                                             lengths, halo, field, s["possrcs"], s["posrecs"]))
        return plan.traces(), plan.field(), files
    finally:
        plan.close()


def solve(lengths, lt, vel, srcs, recs, *, halo, rcoef, ppw, freetop, do_bench, do_vis,
          precision, dt, nt, device, verbose, do_save=False, nsave=5, save_name="snapshot",
          save_dir=os.path.join("simulations", "tmp")):
    if do_vis:
        raise NotImplementedError("do_vis needs a graphics stack, which this build does not have")
    s = prepare(lengths, lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw, freetop=freetop,
                precision=precision, dt=dt, nt=nt)
    p = s["problem"]
    ctx = default_context(device)
    wb = word_bytes(p)
    if do_save and not do_bench:
        traces, pfinal, _ = _run_with_snapshots(ctx, s, lengths, halo, int(nsave), save_name,
                                                save_dir)
        recs.seismograms = traces
        return pfinal
    if do_bench:
        # BenchmarkTools trial of one forward! step (acoustic_3D_xPU.jl:311-353):
        # minimum device time of single-step launches, T_eff from A_eff.
        plan = ctx.plan(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"])
        try:
            times = []
            for _ in range(200):
                if plan.step >= p.nt:
                    plan.reset()
                times.append(plan.run(1, graph=False))
            t_it = min(times) / 1e3
        finally:
            plan.close()
        a_eff = a_eff_words(p) * wb / 1e9
        print(f"size = {_size_str(p)}, time = {t_it:1.3e} sec, Teff = {a_eff / t_it:1.3f} GB/s, "
              f"memory = {alloc_words(p) * wb / 1e9:1.3f} GB")
        return None
    traces = np.zeros((p.nt, p.nrec), order="F")
    pfinal = np.zeros(_shape(p), order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], traces,
                pfinal)
    if verbose and p.nt > 0:
        t_toc = ctx.last_run_ms() / 1e3
        t_it = t_toc / p.nt
        a_eff = a_eff_words(p) * wb / 1e9
        print(f"size = {_size_str(p)}, total time = {t_toc:1.8e} sec, time per it = {t_it:1.8e} "
              f"sec, Teff = {a_eff / t_it if t_it > 0 else 0.0:1.3f} GB/s, "
              f"memory = {alloc_words(p) * wb / 1e9:1.3f} GB")
    recs.seismograms = traces
    return pfinal
