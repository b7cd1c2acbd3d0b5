#!/usr/bin/env python
"""Benchmark of the CPML forward time stepping on B200.

Workload (default): the 3D single-shot case of the headline metric —
256^3 interior + CPML 20 with a free top (296 x 276 x 296 nodes), seeded
smoothed-gradient velocity model, FP32 build, nt = 2000 time steps, 4096
receivers. One benchmark "step" is one shot: state reset + nt time steps.

Metric: T_eff = A_eff / t_timestep in GB/s, with A_eff the reference's
effective-access count (src/shared/acoustic_3D_xPU.jl:520-528) in words of
the computed precision. `value` is measured on device-resident inputs;
`e2e` goes through awc_forward (the drop-in C ABI call) from pinned host
buffers, copies included. Run under torchrun for N GPUs: every rank runs its
own shot (weak scaling, no data-path collective); timing is the max over
ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import datetime
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import __graft_entry__ as G  # noqa: E402


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nt", type=int, default=2000, help="time steps per shot")
    ap.add_argument("--interior", type=int, default=256, help="interior nodes per axis")
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--quick", action="store_true",
                    help="device-resident leg only (no e2e, FP64 or CPU legs); for profiling")
    ap.add_argument("--launch", default=None,
                    help="tile_y,zchunk,band_zchunk of the 3D step instead of autotuning")
    ap.add_argument("--no-oracle", action="store_true",
                    help="skip the full-length error check against the FP64 oracle (~1.5 min "
                         "of host time)")
    ap.add_argument("--blocking", default=None, metavar="DEPTH,ZCHUNKS[,ROWS]",
                    help="fixed time blocking of the 3D leg (default: the autotuner's choice)")
    ap.add_argument("--batch-only", default=None, metavar="TILE_Y,BLOCKS_PER_SM",
                    help="profiling: only the batched 2D workload at --nt steps and this launch "
                         "shape (one eager run, no timing line)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the CPU-baseline sample")
    return ap.parse_args()


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def ncu_value(kernel_tag, key):
    """A `key: value` figure from the committed ncu summary of a kernel."""
    path = os.path.join(ROOT, "profiles", f"ncu_{kernel_tag}.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(re.escape(key) + r":\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def ncu_traffic(kernel_tag):
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"ncu_{kernel_tag}.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id):
        self.bus_id = bus_id
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms",
               "100"]
        if self.bus_id:
            cmd += ["-i", self.bus_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[c - 5] for r in rows for c in range(5, 9)
                          if r[c].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def bus_id_of(dev):
    import torch
    try:
        pr = torch.cuda.get_device_properties(dev)
        return f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        return None


def workload(args):
    pkg = G.load_package()
    from acousticwavecpml_b200 import workloads as W
    w = W.config2(nt=args.nt, interior=args.interior)
    srcs, recs = W.sources_receivers(pkg, w)
    return pkg, w, srcs, recs


def cpu_baseline(w, seconds):
    """The oracle (C++ FP64 OpenMP restatement of the reference's Threads
    path) on a bounded sample of the same shot: the first n time steps."""
    O = G.load_oracle()
    kw = dict(w["kwargs"])
    s = O.setup(w["lengths"], w["lt"], w["vel"], w["src_pos"], w["t0s"], w["f0"], w["rec_pos"],
                **kw)
    p = s["problem"]
    O.forward(s, steps=2)
    per = O.last_loop_seconds() / 2
    n = int(max(3, min(p.nt, seconds / max(per, 1e-6))))
    O.forward(s, steps=n)
    t = O.last_loop_seconds()
    return s, n, t, O.max_threads()


def a_eff(pkg, problem):
    from acousticwavecpml_b200.core import a_eff_words, word_bytes
    return a_eff_words(problem) * word_bytes(problem)


def min_traffic(p):
    """Bytes per 3D time step a perfect kernel must move: 4 words per interior
    node (read pold, pcur, fact; write pnew) plus, per active CPML side, one
    read and one write of every ψ (h+1 layers) and ξ (h layers) entry. The
    free top leaves one y side inactive."""
    from acousticwavecpml_b200.core import word_bytes
    w = word_bytes(p)
    active_sides = (2, 1 if p.freetop else 2, 2)
    n = [p.nx - 2, p.ny - 2, p.nz - 2]
    cells = n[0] * n[1] * n[2]
    band = 0
    for a in range(3):
        cross = cells // n[a]
        band += active_sides[a] * 2 * ((p.halo + 1) + p.halo) * cross
    return w * (4 * cells + band)


def interior_cells(p):
    return (p.nx - 2) * (p.ny - 2) * ((p.nz - 2) if p.ndim == 3 else 1)


def run_reference(args):
    """--impl reference: the reference's CPU path, restated (Julia is not
    available), FP64 on all host cores; each step is a bounded sample."""
    pkg, w, srcs, recs = workload(args)
    O = G.load_oracle()
    s = O.setup(w["lengths"], w["lt"], w["vel"], w["src_pos"], w["t0s"], w["f0"], w["rec_pos"],
                **w["kwargs"])
    p = s["problem"]
    O.forward(s, steps=2)
    per = O.last_loop_seconds() / 2
    n = int(max(2, min(p.nt, 8.0 / max(per, 1e-6))))  # ~8 s per step
    for _ in range(args.warmup):
        O.forward(s, steps=min(n, 2))
    tot = 0.0
    for _ in range(args.steps):
        O.forward(s, steps=n)
        tot += O.last_loop_seconds()
    t_step = tot / (args.steps * n)
    ab = a_eff(pkg, p)
    val = ab / t_step / 1e9
    line = {
        "impl": "reference", "metric": "3D T_eff GB/s vs HBM peak", "value": val, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded smoothed-gradient model)",
        "config": {"workload": w["name"], "grid": [p.nx, p.ny, p.nz], "nt": p.nt,
                   "halo": p.halo, "freetop": True,
                   "sample": f"first {n} of {p.nt} time steps per step"},
        "gcells_per_s": interior_cells(p) / t_step / 1e9,
        "cpu_baseline": {"value": val, "unit": "GB/s", "cores": O.max_threads(), "kind": "port",
                         "sample": f"{n} time steps of {w['name']} per step, FP64, "
                                   "C++/OpenMP restatement of the Threads path"},
        "e2e": {"value": val, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch_leg(pkg, ctx, args, rank, world, timed, peak, keep=None):
    """Batched 2D shots, FP32: the 96 shots of the six-model layered workload,
    rank r taking shots r, r + N, ... (no data-path collective). One step of
    this leg = every shot of the rank's batch advanced over all nt time steps
    (one CUDA graph replay); time = max over ranks."""
    from acousticwavecpml_b200 import workloads as W
    w = W.config3()
    shots = W.batch_shots(pkg, w)
    mine = pkg.batch.shard(shots, rank, world)
    probs, vels, setups, idx = pkg.prepare_batch(w["models"], mine, **w["kwargs"])
    b = pkg.Batch(ctx, probs, vels, setups, idx)
    b.autotune(20)
    nt = b.nt

    def run():
        b.reset()
        b.run(nt, graph=True)

    run()
    k = 2
    ms = timed(run, k)
    words = sum(pkg.core.a_eff_words(st["problem"]) for st in setups)
    nodes = sum(st["problem"].nx * st["problem"].ny for st in setups)
    t_ts = ms / 1e3 / (k * nt)
    ty, bps = b.get_launch()
    if keep is not None:  # traces of the first shot of each model (for the oracle check)
        first = {}
        for g, sh in enumerate(w["shots"]):
            first.setdefault(sh["model"], g)
        for g in first.values():
            if g % world == rank:
                keep[g] = (w, b.traces(g // world))
    b.close()
    achieved = words * 4 / t_ts / 1e9
    traffic = ncu_traffic("step2d_batch_tma_96shots") if world == 1 else None
    l2_bytes = ncu_value("step2d_batch_tma_96shots", "l2_bytes_per_launch") if world == 1 else None
    dram = None
    if traffic:
        dram = {"traffic_bytes_per_step": traffic, "achieved": traffic / t_ts / 1e9,
                "frac": traffic / t_ts / 1e9 / peak,
                "note": "real DRAM bytes (ncu, profiles/) per step over the measured step time: "
                        "the 16 shots of a model share fact and the small models' fields "
                        "partly stay in the 126 MB L2, so A_eff over-counts DRAM traffic"}
    return {"workload": w["name"], "shots": len(shots), "models": len(w["models"]),
            "nt": nt, "dtype": "f32", "value": len(shots) / (ms / 1e3 / k), "unit": "shots/s",
            "us_per_timestep": t_ts * 1e6, "gnodes_per_s": world * nodes / t_ts / 1e9,
            "t_eff_gbs": world * achieved,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "per_launch": "one time step of every shot of the rank's batch = one "
                                       "persistent batched-step launch; A_eff summed over "
                                       "shots, FP32 words"},
            "dram_roofline": dram,
            "l2": ({"traffic_bytes_per_step": l2_bytes, "achieved_gbs": l2_bytes / t_ts / 1e9,
                    "note": "ncu lts__t_bytes of one step (profiles/) over the measured step "
                            "time; no measured L2 peak on this pool, so no fraction"}
                   if l2_bytes else None),
            "launch": {"tile": [64 if ty <= 16 else 32, ty], "blocks_per_sm": bps,
                       "kernel": "step2d_batch_tma (TMA stages, producer warp)" if ty <= 16
                                 else "step2d_batch (register strips)"},
            "gpu_launches": k * nt, "timed_runs": k,
            "sharding": f"shots {rank}::{world} per rank" if world > 1 else "one batch"}


def oracle_check(pkg, ctx, w2, traces32, traces64, pend64, batch_traces):
    """Relative L2 errors against the FP64 oracle at full length: config 1
    (2D, 241 x 241, nt = 1000, FP64 and FP32 through awc_forward), config 2
    (the headline shot, nt = 2000: the timed FP32 run's traces and the FP64
    build's traces and final field), config 3 (the first shot of each of the
    six models of the batched run, nt = 3000, FP32)."""
    from acousticwavecpml_b200 import workloads as W
    O = G.load_oracle()

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))

    out = {"tolerance": {"f64": 1e-10, "f32_traces": 1e-4}}
    w1 = W.config1()
    so = O.setup(w1["lengths"], w1["lt"], w1["vel"], w1["src_pos"], w1["t0s"], w1["f0"],
                 w1["rec_pos"], **w1["kwargs"])
    pe_o, tr_o = O.forward(so)
    srcs, recs = W.sources_receivers(pkg, w1)
    for prec in ("f64", "f32"):
        s = pkg.prepare(w1["lengths"], w1["lt"], w1["vel"], srcs, recs, precision=prec,
                        **w1["kwargs"])
        p = s["problem"]
        tr = np.zeros((p.nt, p.nrec), order="F")
        pe = np.zeros(s["vel"].shape, order="F")
        ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr, pe)
        out[f"config1_{prec}"] = {"traces": rel(tr, tr_o), "field": rel(pe, pe_o)}
    so = O.setup(w2["lengths"], w2["lt"], w2["vel"], w2["src_pos"], w2["t0s"], w2["f0"],
                 w2["rec_pos"], **w2["kwargs"])
    pe_o, tr_o = O.forward(so)
    out["config2_f32"] = {"traces": rel(traces32, tr_o)}
    if traces64 is not None:
        out["config2_f64"] = {"traces": rel(traces64, tr_o), "field": rel(pend64, pe_o)}
    for k, (w3, tr) in sorted(batch_traces.items()):
        sh = w3["shots"][k]
        kw = w3["kwargs"]
        lx, ly, vel = w3["models"][sh["model"]]
        dt = pkg.prepare((lx, ly), None, vel,
                         pkg.Sources(sh["src_pos"], sh["t0s"], [pkg.rickersource1D], sh["f0"]),
                         pkg.Receivers(sh["rec_pos"]), **kw)["dt"]
        so = O.setup((lx, ly), None, vel, sh["src_pos"], sh["t0s"], sh["f0"], sh["rec_pos"],
                     halo=kw["halo"], rcoef=kw["rcoef"], freetop=True, dt=dt, nt=kw["nt"])
        _, tr_o = O.forward(so)
        out[f"config3_model{sh['model']}_shot{k}_f32"] = {"traces": rel(tr, tr_o)}
    return out


def batch_profile_run(args, local):
    """--batch-only: the batched 2D workload at args.nt steps with a fixed
    launch shape, run once eagerly (one launch per step), for ncu."""
    pkg = G.load_package()
    from acousticwavecpml_b200 import workloads as W
    w = W.config3(nt=args.nt)
    probs, vels, setups, idx = pkg.prepare_batch(w["models"], W.batch_shots(pkg, w), **w["kwargs"])
    b = pkg.Batch(pkg.Context(local), probs, vels, setups, idx)
    ty, bps = (int(x) for x in args.batch_only.split(","))
    b.set_launch(ty, bps)
    b.run(args.nt, graph=False)
    print(json.dumps({"batch_only": w["name"], "launch": [ty, bps], "steps": b.step}))
    b.close()


def gradient_leg(pkg, ctx, rank, world, timed_host):
    """3D gradient, FP32 with an FP64 check: config 4's 16 shots, dJ/d(c²)
    summed over the shots at the initial model against the true model's
    traces of the same precision, through awc_misfit_gradient_shots (host
    buffers, checkpoint every 50 steps, nt = 1500; one call per rank, the
    shots' gradients summed on the device). Rank r takes shots r, r + N, ...;
    under torchrun the ranks' sums are added with one all-reduce
    (adjoint.sharded_gradient). Also timed: one awc_misfit_gradient call per
    shot for two shots. The FP64 build checks shot 0."""
    import time
    import torch
    import torch.distributed as dist
    from acousticwavecpml_b200 import adjoint
    from acousticwavecpml_b200 import workloads as W
    w = W.config4()
    R = pkg.Receivers(w["rec_pos"])
    kw = dict(w["kwargs"])
    nshot = len(w["shots"])

    def setups(shot, precision):
        S = pkg.Sources(w["shots"][shot], w["t0s"], [pkg.rickersource1D], w["f0"])
        st = pkg.prepare(w["lengths"], None, w["true"], S, R, precision=precision, **kw)
        si = pkg.prepare(w["lengths"], None, w["init"], S, R, precision=precision, **kw)
        si["coeffs"] = st["coeffs"]  # the CPML profile of the true model's vmax
        p = st["problem"]
        obs = np.zeros((p.nt, p.nrec), order="F")
        ctx.forward(p, st["vel"], st["coeffs"], st["possrcs"], st["dt2srctf"], st["posrecs"], obs)
        return st, si, obs

    # observed data of every shot of this rank (not timed)
    mine = list(range(rank, nshot, world))
    data = {k: setups(k, "f32") for k in (mine or [0])}
    st0, si0, obs0 = data[(mine or [0])[0]]
    p = st0["problem"]
    t0 = time.perf_counter()
    ctx.forward(p, si0["vel"], si0["coeffs"], si0["possrcs"], si0["dt2srctf"], si0["posrecs"],
                np.zeros((p.nt, p.nrec), order="F"))
    t_fwd = time.perf_counter() - t0
    adjoint.misfit_gradient(si0, obs0, w["checkpoint_every"], ctx)  # warm-up

    # the rank's shots share one velocity array, and their observed traces
    # are stacked (nt x nrec x shots) before the timed region
    for k in mine:
        data[k][1]["vel"] = si0["vel"]
    obs_all = np.asfortranarray(np.stack([data[k][2] for k in mine], axis=-1)) if mine else None

    def shots_of(ks):
        return adjoint.misfit_gradient_shots([data[k][1] for k in ks],
                                             obs_all if ks == mine else [data[k][2] for k in ks],
                                             w["checkpoint_every"], ctx)

    out = {}
    t_grad = timed_host(lambda: out.update(
        r=adjoint.sharded_gradient(list(range(nshot)), shots_of, w["init"].shape,
                                   batched=True)))
    J32_all, g32_all = out["r"]
    # one call per shot (rank 0's first two shots), for comparison
    k2 = (mine or [0])[:2]
    t0 = time.perf_counter()
    for k in k2:
        adjoint.misfit_gradient(data[k][1], data[k][2], w["checkpoint_every"], ctx)
    t_single = (time.perf_counter() - t0) / len(k2)
    # FP64 check on shot 0 (rank 0), against its own FP64 data; and the FP32
    # adjoint given the FP64 residual, which separates the adjoint's own
    # rounding from the residual's (a small difference of two FP32 traces)
    res = {}
    if rank == 0:
        J32, g32, tr32 = adjoint.misfit_gradient(si0, obs0, w["checkpoint_every"], ctx)
        _, s64, obs64 = setups(0, "f64")
        s64["coeffs"] = si0["coeffs"]
        J64, g64, tr64 = adjoint.misfit_gradient(s64, obs64, w["checkpoint_every"], ctx)
        inj = np.asfortranarray(tr32 - (tr64 - obs64))
        _, g32i, _ = adjoint.misfit_gradient(si0, inj, w["checkpoint_every"], ctx)
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
        res = {"fp32_vs_fp64_gradient_rel_l2": rel(g32, g64),
               "fp32_vs_fp64_misfit_rel": abs(J32 - J64) / J64,
               "fp32_vs_fp64_residual_rel_l2": rel(tr32 - obs0, tr64 - obs64),
               "fp32_adjoint_on_fp64_residual_vs_fp64_gradient_rel_l2": rel(g32i, g64)}
    return {"workload": w["name"], "dtype": "f32", "shots": nshot, "shots_per_rank": len(mine),
            "value": nshot / t_grad, "unit": "shot gradients/s",
            "s_for_all_shots": t_grad, "s_per_gradient": t_grad * world / nshot,
            "s_per_forward": t_fwd, "gradient_over_forward": t_grad * world / nshot / t_fwd,
            "s_per_gradient_one_call_per_shot": t_single,
            "one_call_per_shot_over_forward": t_single / t_fwd,
            "misfit_all_shots": float(J32_all), "checkpoint_every": w["checkpoint_every"],
            "nt": p.nt, "grid": [p.nx, p.ny, p.nz], **res,
            "check_shot": 0,
            "timing": "host wall clock of the per-shot C-ABI calls (uploads, checkpointed "
                      "forward, recompute, adjoint, download) and the summation (one all-reduce "
                      "under torchrun), max over ranks"}


def learned_leg(pkg, ctx):
    """The learned 4-node layer against the 20-node CPML at config 5's grid
    sizes (384^3 interior, free top; CPML-20 on 424 x 404 x 424, learned-4 on
    392 x 388 x 392): device time per step of one shot each (CUDA events
    around the time loop inside awc_forward_learned and awc_forward; nt = 120,
    a seeded layered velocity model in 1500-4500 m/s, the MLP with seeded
    random BF16 weights). Speed only: no learned layer is accepted (every
    trained candidate is unstable), so no reflected energy is measured."""
    from acousticwavecpml_b200 import learned as L
    rng = np.random.default_rng(55)
    n, nt, d = 384, 120, 10.0
    out = {"workload": "learned4_vs_cpml20_384cube_1shot_nt120", "nt": nt}
    for name, halo, learned in (("cpml20", 20, False), ("learned4", 4, True)):
        shape = (n + 2 * halo, n + halo, n + 2 * halo)
        tops = np.sort(rng.integers(1, shape[1] - 1, 5))
        layer_c = 1500.0 + 3000.0 * np.sort(rng.random(6))
        cy = layer_c[np.searchsorted(tops, np.arange(shape[1]))]
        vel = np.asfortranarray(np.broadcast_to(cy[None, :, None], shape)
                                * (1.0 + 0.02 * rng.standard_normal(shape)))
        S = pkg.Sources([[(shape[0] // 2) * d, (halo + 10) * d, (shape[2] // 2) * d]], [0.04],
                        [pkg.rickersource1D], 10.0)
        R = pkg.Receivers([[(halo + 5 + 12 * i) * d, (halo + 5) * d, (shape[2] // 2) * d]
                           for i in range(30)])
        s = pkg.prepare(tuple((m - 1) * d for m in shape), None, vel, S, R, halo=halo, ppw=1e-9,
                        freetop=True, precision="f32", nt=nt)
        p = s["problem"]
        if learned:
            k = L.n_inputs(3)
            wb = L.to_bf16(L.pack(rng.standard_normal((32, k)) / np.sqrt(k),
                                  0.05 * rng.standard_normal(32),
                                  rng.standard_normal((32, 32)) / np.sqrt(32),
                                  0.05 * rng.standard_normal(32),
                                  rng.standard_normal(32) / np.sqrt(32) * 0.3, 0.01))
            run = lambda: L.forward_learned(s, wb, ctx)  # noqa: E731
        else:
            tr = np.zeros((p.nt, p.nrec), order="F")
            run = lambda: ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"],  # noqa: E731
                                      s["dt2srctf"], s["posrecs"], tr)
        run()  # warm-up (and the CPML plan's autotuning)
        ms = []
        for _ in range(3):
            run()
            ms.append(ctx.last_run_ms())
        out[f"{name}_grid"] = list(shape)
        out[f"{name}_us_per_step"] = 1e3 * min(ms) / nt
    out["learned_speedup"] = out["cpml20_us_per_step"] / out["learned4_us_per_step"]
    out["target_speedup"] = 1.3
    out["tensor_pipe_active_pct"] = ncu_value("learned_layer_3d_168x164x168",
                                              "tensor_pipe_active_pct")
    out["accepted"] = False
    return out


def main():
    args = parse_args()
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    if args.batch_only:
        batch_profile_run(args, local)
        return
    pkg, w, srcs, recs = workload(args)
    s = pkg.prepare(w["lengths"], w["lt"], w["vel"], srcs, recs, precision=args.precision,
                    **w["kwargs"])
    p = s["problem"]
    nt = p.nt
    ctx = pkg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))

    def timed(fn, k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # ---- device-resident leg ------------------------------------------------
    plan = ctx.plan(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"])
    if args.launch:
        plan.set_launch(*[int(x) for x in args.launch.split(",")])
    else:
        plan.autotune(120)  # launch shape picked on this data, before any timing
    if args.blocking:
        plan.set_blocking(*[int(x) for x in args.blocking.split(",")])
    launch = plan.get_launch()
    depth, tb_zchunks, tb_rows = plan.get_blocking()

    def shot():
        plan.reset()
        plan.run(nt, graph=True)

    for _ in range(max(args.warmup, 0)):
        shot()
    with ClockSampler(bus_id_of(local)) as clk:
        ms = timed(shot, args.steps)
    clocks = clk.summary()
    traces_dev = plan.traces()
    plan.reset()
    launches = args.steps * plan.launch_count(nt)
    plan.close()

    ab = a_eff(pkg, p)
    t_ts = ms / 1e3 / (args.steps * nt)  # seconds per time step (this rank's max)
    value = world * ab / t_ts / 1e9
    peak, peak_src = measured_peak()
    tag = f"step3d_{args.precision}_{p.nx}x{p.ny}x{p.nz}"
    traffic = ncu_traffic(tag)
    achieved = ab / t_ts / 1e9
    line = {
        "metric": "3D T_eff GB/s vs HBM peak", "value": value, "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic (seeded smoothed-gradient velocity model, Ricker source)",
        "config": {"workload": w["name"], "grid": [p.nx, p.ny, p.nz], "nt": nt, "halo": p.halo,
                   "freetop": True, "nrec": p.nrec, "precision": args.precision,
                   "step": "one shot = state reset + nt fused time steps (CUDA graph)",
                   "l2": "inputs larger than L2 (4 fields of "
                         f"{p.nx * p.ny * p.nz * (4 if args.precision == 'f32' else 8) / 1e6:.1f}"
                         " MB each, no flush needed)",
                   "parallelism": f"shots{world}",
                   "launch": {"core_tile": [64, launch[0]], "core_zchunk": launch[1],
                              "band_zchunk": launch[2], "depth": depth,
                              "depth2_zchunks": tb_zchunks, "depth2_rows": tb_rows}},
        "gcells_per_s": world * interior_cells(p) / t_ts / 1e9,
        "us_per_timestep": t_ts * 1e6,
        "a_eff_bytes_per_timestep": ab,
        "min_traffic_bytes_per_timestep": min_traffic(p),
        "a_eff_over_min_traffic": ab / min_traffic(p),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src,
                     "per_launch": "one time step: at depth 1 two kernel launches over "
                                   "disjoint nodes (the band-free core box and the CPML "
                                   "band boxes, parallel graph branches, sources and "
                                   "receivers fused), at depth 2 half of one two-step pass; "
                                   "achieved = A_eff of one step / CUDA-event time per step "
                                   "of the graph replays; traffic = ncu DRAM bytes of one "
                                   "step (both kernels)"},
        "gpu_launches": launches,
        "clocks": clocks,
    }

    if not args.quick:
        # ---- end-to-end through the C ABI from pinned host buffers ----------
        vel_h = torch.empty(s["vel"].size, dtype=torch.float64, pin_memory=True)
        vel_h.numpy()[:] = s["vel"].ravel(order="F")
        tr_h = torch.empty(nt * p.nrec, dtype=torch.float64, pin_memory=True)
        pf_h = torch.empty(s["vel"].size, dtype=torch.float64, pin_memory=True)

        def e2e_call():
            ctx.forward(p, vel_h, s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr_h,
                        pf_h)

        for _ in range(max(args.warmup, 1)):
            e2e_call()
        ms_e2e = timed(e2e_call, args.steps)
        tr_e2e = tr_h.numpy().reshape((nt, p.nrec), order="F")
        h2d = (s["vel"].nbytes + s["coeffs"].nbytes + s["possrcs"].nbytes + s["dt2srctf"].nbytes +
               s["posrecs"].nbytes)
        d2h = tr_h.numel() * 8 + pf_h.numel() * 8
        line["e2e"] = {"value": world * ab * nt / (ms_e2e / 1e3 / args.steps) / 1e9,
                       "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "ms_per_step": ms_e2e / args.steps,
                       "call": "awc_forward (host buffers, pinned)"}
        line["e2e_matches_device_leg"] = bool(np.array_equal(tr_e2e, traces_dev))

        # ---- FP64 build of the same shot (parity build), device-resident ----
        if args.precision == "f32":
            s64 = pkg.prepare(w["lengths"], w["lt"], w["vel"], srcs, recs, precision="f64",
                              **w["kwargs"])
            p64 = s64["problem"]
            plan64 = ctx.plan(p64, s64["vel"], s64["coeffs"], s64["possrcs"], s64["dt2srctf"],
                              s64["posrecs"])

            def shot64():
                plan64.reset()
                plan64.run(nt, graph=True)

            plan64.autotune(10)
            shot64()
            k64 = max(1, min(args.steps, 3))
            ms64 = timed(shot64, k64)
            tr64 = plan64.traces()
            pe64 = plan64.field()
            plan64.close()
            t64 = ms64 / 1e3 / (k64 * nt)
            ab64 = a_eff(pkg, p64)
            line["fp64"] = {"value": world * ab64 / t64 / 1e9, "unit": "GB/s",
                            "gcells_per_s": world * interior_cells(p64) / t64 / 1e9,
                            "us_per_timestep": t64 * 1e6, "frac": ab64 / t64 / 1e9 / peak}
            nrm = np.linalg.norm(tr64)
            line["fp32_vs_fp64_traces_rel_l2"] = float(np.linalg.norm(traces_dev - tr64) /
                                                       (nrm if nrm > 0 else 1.0))

        # ---- batched 2D shots (96 shots over 6 layered models), sharded -----
        batch_traces = {}
        line["batch"] = batch_leg(pkg, ctx, args, rank, world, timed, peak, batch_traces)

        # ---- 3D gradient by the discrete adjoint (one shot per rank) -------
        def timed_host(fn):
            import time
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            fn()
            t = time.perf_counter() - t0
            if world > 1:
                tt = torch.tensor([t], device="cuda")
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                t = float(tt.item())
            return t

        line["gradient"] = gradient_leg(pkg, ctx, rank, world, timed_host)
        if world == 1:
            line["learned"] = learned_leg(pkg, ctx)

        # ---- full-length errors against the FP64 oracle (N=1) -------------
        if world == 1 and rank == 0 and not args.no_oracle:
            f64 = args.precision == "f32"
            line["err_vs_oracle"] = oracle_check(pkg, ctx, w, traces_dev,
                                                 tr64 if f64 else None, pe64 if f64 else None,
                                                 batch_traces)

        # ---- CPU baseline (rank 0 at N=1 only) ------------------------------
        if world == 1 and rank == 0:
            so, n, t, cores = cpu_baseline(w, args.cpu_seconds)
            t_cpu = t / n
            ab_cpu = a_eff(pkg, so["problem"])
            line["cpu_baseline"] = {
                "value": ab_cpu / t_cpu / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
                "sample": f"first {n} of {nt} time steps of {w['name']}, FP64, C++/OpenMP "
                          "restatement of the reference Threads path (Julia absent)",
                "gcells_per_s": interior_cells(so["problem"]) / t_cpu / 1e9,
                "s_per_timestep": t_cpu}
            if "fp64" in line:
                # like for like: the FP64 build against the FP64 CPU port, per cell update
                line["fp64"]["vs_cpu_baseline_gcells"] = (line["fp64"]["gcells_per_s"] /
                                                          line["cpu_baseline"]["gcells_per_s"])

    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
