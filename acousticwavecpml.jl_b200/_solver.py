"""Shared body of solve2D/solve3D: setup, one awc_forward call, outputs."""
import numpy as np

from .core import a_eff_words, alloc_words, default_context, prepare, word_bytes


def _size_str(problem):
    if problem.ndim == 2:
        return f"{problem.nx}x{problem.ny}"
    return f"{problem.nx}x{problem.ny}x{problem.nz}"


def solve(lengths, lt, vel, srcs, recs, *, halo, rcoef, ppw, freetop, do_bench, do_vis,
          precision, dt, nt, device, verbose):
    if do_vis:
        raise NotImplementedError("do_vis needs a graphics stack, which this build does not have")
    s = prepare(lengths, lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw, freetop=freetop,
                precision=precision, dt=dt, nt=nt)
    p = s["problem"]
    ctx = default_context(device)
    wb = word_bytes(p)
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
    pfinal = np.zeros(s["vel"].shape, order="F")
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
