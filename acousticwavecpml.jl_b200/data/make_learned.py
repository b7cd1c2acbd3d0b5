"""Trains the 2D learned thin layer (width 4) and measures it against CPML-20.

    python acousticwavecpml.jl_b200/data/make_learned.py [out_dir]

Needs a GPU. Writes learned2d_w4.npz (BF16 weights) and learned2d_w4.json
(training loss, and for held-out models the reflected energy of the learned
layer and of a CPML-20 band against a reflection-free reference) to out_dir
(default: this folder).

Cases are seeded synthetic 2D models on a 200 x 150 core region (dx = 10 m,
free top): homogeneous or layered velocities in 1500..4500 m/s, one Ricker
source in the core (f0 in 8..14 Hz), nt = 1000 steps at the CFL time step of
the model. Training inputs come from reflection-free reference runs: the
same model padded by 300 nodes on every absorbing side. Candidates: a
least-squares linear layer and an MLP fitted to one-step targets, and both
fine-tuned through 100-step windows of the layer scheme (torch autograd);
the candidate with the smallest worst-case reflected energy on the held-out
models is kept.
"""
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CORE = (200, 150)
DX = 10.0
WIDTH = 4
NT = 1000


def core_model(rng):
    nx, ny = CORE
    if rng.random() < 0.3:
        return np.full((nx, ny), float(rng.uniform(1500.0, 4500.0)))
    nint = int(rng.integers(1, 5))
    depths = np.sort(rng.choice(np.arange(10, ny - 10), size=nint, replace=False))
    v = np.sort(rng.uniform(1500.0, 4500.0, size=nint + 1))
    col = np.full(ny, v[0])
    for k, j in enumerate(depths):
        col[j:] = v[k + 1]
    return np.repeat(col[None, :], nx, axis=0)


def grid_model(core, band):
    """The core model extended by `band` absorbing nodes plus the rim on the
    left, right and bottom (edge values repeated); returns (model, x offset
    of the core in nodes)."""
    off = band + 1
    return np.asfortranarray(np.pad(core, ((off, off), (0, off)), mode="edge")), off


def make_case(pkg, rng):
    core = core_model(rng)
    cmax = float(core.max())
    f0 = float(rng.uniform(8.0, 14.0))
    dt = math.sqrt(2.0) / (cmax * (2.0 / DX)) / 2.0
    sx = float(rng.uniform(20, CORE[0] - 20)) * DX
    sy = float(rng.uniform(5, CORE[1] - 20)) * DX
    rec = [[i * DX, j * DX] for i in range(0, CORE[0], 4) for j in range(1, CORE[1], 4)]
    return dict(core=core, f0=f0, t0=1.2 / f0, dt=dt, src=[[sx, sy]], rec=rec)


def setup(pkg, case, band, precision):
    """prepare() of the case on a grid with `band` absorbing nodes, positions
    shifted into that grid."""
    vel, off = grid_model(case["core"], band)
    L = ((vel.shape[0] - 1) * DX, (vel.shape[1] - 1) * DX)
    shift = np.array([off * DX, 0.0])
    S = pkg.Sources(np.asarray(case["src"]) + shift, [case["t0"]], [pkg.rickersource1D],
                    case["f0"])
    R = pkg.Receivers(np.asarray(case["rec"]) + shift)
    s = pkg.prepare(L, None, vel, S, R, halo=band, rcoef=1e-4, ppw=1e-9, freetop=True,
                    precision=precision, dt=case["dt"], nt=NT)
    return s, L, vel, S, R


def traces(pkg, ctx, s):
    p = s["problem"]
    tr = np.zeros((p.nt, p.nrec), order="F")
    ctx.forward(p, s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"], s["posrecs"], tr)
    return tr


def main(out_dir):
    import __graft_entry__ as g
    pkg = g.load_package()
    from acousticwavecpml_b200 import learned
    ctx = pkg.default_context(0)
    rng = np.random.default_rng(2026)
    log = []

    def say(msg):
        print(msg, flush=True)
        log.append(msg)

    t0 = time.time()
    train_cases = [make_case(pkg, rng) for _ in range(16)]
    test_cases = [make_case(pkg, rng) for _ in range(4)]
    data = []
    for c in train_cases:
        s, L, vel, S, R = setup(pkg, c, WIDTH, "f64")
        data.append(dict(lengths=L, vel=vel, srcs=S, recs=R, dt=c["dt"], nt=NT, freetop=True))
    X, Y = learned.training_data(pkg, data, width=WIDTH, pad=300, keep=0.25, ctx=ctx)
    say(f"training samples {len(X)} ({time.time() - t0:.0f} s)")
    # candidate layers: least squares (linear) and an MLP fitted step by step,
    # then both fine-tuned through 100-step windows of the scheme itself
    import torch
    base = {"linear": learned.fit_linear(X, Y),
            "mlp": learned.train(X, Y, epochs=10, log=say)}
    n_samples = int(len(X))
    del X, Y
    sims, refs = [], []
    for c, dd in zip(train_cases[:8], data[:8]):
        s, *_ = setup(pkg, c, WIDTH, "f32")
        node = [int(v) - 1 for v in s["possrcs"][0]]
        sims.append(learned.RolloutSim(dd["vel"], c["dt"], (DX, DX), WIDTH, True, node,
                                       s["dt2srctf"][:, 0]))
        R = [np.zeros(dd["vel"].shape[::-1], dtype=np.float32)]
        for _, pnew in learned.reference_fields(pkg, dd["lengths"], dd["vel"], dd["srcs"],
                                                dd["recs"], dt=c["dt"], nt=NT, width=WIDTH,
                                                ctx=ctx):
            R.append(pnew.T.astype(np.float32))
        refs.append(torch.tensor(np.stack(R), device="cuda"))
    say(f"rollout cases ready ({time.time() - t0:.0f} s)")
    for name in ("linear", "mlp"):
        base[name + "_rollout"] = learned.train_rollout(base[name], sims, refs, iters=600,
                                                        lr=3e-4, log=say)
        say(f"{name} rollout done ({time.time() - t0:.0f} s)")
    cands = {}
    for name, flat in base.items():
        for gamma in (0.0, 0.02, 0.05):
            cands[f"{name}_g{gamma}"] = learned.to_bf16(learned.damped(flat, gamma, 2))
    report = dict(width=WIDTH, core=CORE, dx=DX, nt=NT, samples=n_samples, cases=[],
                  candidates=sorted(cands))
    scores = {k: [] for k in cands}
    for n, c in enumerate(test_cases):
        # reference: the model padded so far that nothing reflects back in time
        sref, *_ = setup(pkg, c, 320, "f64")
        ref = traces(pkg, ctx, sref)
        s20, *_ = setup(pkg, c, 20, "f32")
        e20 = learned.reflected_energy(traces(pkg, ctx, s20), ref)
        s4c, *_ = setup(pkg, c, WIDTH, "f32")  # a plain 4-node CPML for scale
        e4c = learned.reflected_energy(traces(pkg, ctx, s4c), ref)
        row = dict(cpml20=e20, cpml4=e4c, f0=c["f0"], cmax=float(c["core"].max()),
                   cmin=float(c["core"].min()))
        for name, wb in cands.items():
            tr4, _ = learned.forward_learned(s4c, wb, ctx)
            e = learned.reflected_energy(tr4, ref) if np.all(np.isfinite(tr4)) else float("inf")
            row[name] = e
            scores[name].append(e)
        say(f"test {n}: CPML-20 {e20:.3e}, CPML-4 {e4c:.3e}, " +
            ", ".join(f"{k} {row[k]:.2e}" for k in sorted(cands)))
        report["cases"].append(row)
    best = min(cands, key=lambda k: max(scores[k]))
    wb = cands[best]
    report["chosen"] = best
    say(f"chosen: {best} (worst case {max(scores[best]):.3e})")
    report["log"] = log
    os.makedirs(out_dir, exist_ok=True)
    np.savez(os.path.join(out_dir, "learned2d_w4.npz"), w_bf16=wb)
    with open(os.path.join(out_dir, "learned2d_w4.json"), "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
