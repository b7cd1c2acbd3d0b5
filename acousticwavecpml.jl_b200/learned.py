"""Learned thin absorbing layer (awc_forward_learned in include/awcpml.h).

The CPML band of width 20 is replaced by a layer of W nodes (4 by default)
whose new values come from a small MLP over the 3^d block of nodes around
each layer node at the three latest time levels (see the header comment of
csrc/awc_learned.cu for the exact input layout). This module holds:
  * forward_learned: the solve through the C ABI;
  * layer_nodes / gather: the input layout, restated on the host so that
    training inputs match the kernel's exactly;
  * training_data: inputs and targets from reflection-free reference runs (the
    same model on a grid padded by `pad` nodes, whose outer boundary is so far
    that nothing it reflects reaches the small grid within nt steps);
  * train: fits the MLP (torch, float32, weights rounded to BF16 at the end);
  * reflected_energy: the interior error energy of a solve against the padded
    reference, the figure that decides whether a layer beats CPML-20.
The reference has no counterpart; its absorbing boundary is the CPML.
"""
import ctypes
import math
import os

import numpy as np

from . import _lib
from ._lib import check
from .core import _ptr, default_context, prepare

HIDDEN = 32
DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def n_inputs(ndim):
    """3 time levels x 3^d nodes, plus the local Courant number."""
    return 28 if ndim == 2 else 82


def courant(vel, dt, d, coords, ax):
    """c dt / d along each layer node's normal axis (the kernel forms it as
    sqrt(F) / d with F = dt² c² in FP32)."""
    ndim = vel.ndim
    c = vel[tuple(coords[:, a] for a in range(ndim))]
    dd = np.asarray(d, dtype=np.float64)[ax]
    F = (dt * dt * c.astype(np.float64) ** 2).astype(np.float32).astype(np.float64)
    return np.sqrt(F) / dd


def weights_len(ndim):
    k = n_inputs(ndim)
    return HIDDEN * k + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN + 1


def to_bf16(w):
    """float array -> BF16 bit patterns (uint16), round to nearest even."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    u = w.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def from_bf16(b):
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([np.ravel(W1), np.ravel(b1), np.ravel(W2), np.ravel(b2),
                           np.ravel(W3), np.ravel([b3])]).astype(np.float32)


def unpack(flat, ndim):
    k = n_inputs(ndim)
    f = np.asarray(flat, dtype=np.float32)
    o = 0
    W1 = f[o:o + HIDDEN * k].reshape(HIDDEN, k); o += HIDDEN * k
    b1 = f[o:o + HIDDEN]; o += HIDDEN
    W2 = f[o:o + HIDDEN * HIDDEN].reshape(HIDDEN, HIDDEN); o += HIDDEN * HIDDEN
    b2 = f[o:o + HIDDEN]; o += HIDDEN
    W3 = f[o:o + HIDDEN]; o += HIDDEN
    b3 = f[o]
    return W1, b1, W2, b2, W3, b3


def load_weights(name="learned2d_w4"):
    """BF16 weights shipped with the package (uint16 array)."""
    return np.load(os.path.join(DATA, name + ".npz"))["w_bf16"]


def forward_learned(s, weights_bf16, ctx=None):
    """Solve the shot set up in `s` (prepare() with precision "f32" and halo =
    the layer width) with the learned layer; returns (traces, final field)."""
    ctx = ctx or default_context()
    p = s["problem"]
    w = np.ascontiguousarray(weights_bf16, dtype=np.uint16)
    if w.size != weights_len(p.ndim):
        raise ValueError(f"need {weights_len(p.ndim)} BF16 weights for ndim={p.ndim}")
    traces = np.zeros((p.nt, p.nrec), order="F")
    pfinal = np.zeros(s["vel"].shape, order="F")
    check(_lib.lib().awc_forward_learned(ctx.handle, ctypes.byref(p), _ptr(s["vel"]), _ptr(w),
                                         _ptr(s["possrcs"]), _ptr(s["dt2srctf"]),
                                         _ptr(s["posrecs"]), _ptr(traces), _ptr(pfinal)),
          ctx.handle)
    return traces, pfinal


# ---- input layout -----------------------------------------------------------

def layer_nodes(shape, width, freetop):
    """Layer nodes of a grid (0-based (i, j[, k]) rows), with the axis and
    outward sign of the nearest absorbing side (the kernel's rule: the
    smallest distance to an absorbing side, x before y before z, left before
    right on ties)."""
    ndim = len(shape)
    grids = np.meshgrid(*[np.arange(1, n - 1) for n in shape], indexing="ij")
    coords = np.stack([g.ravel(order="F") for g in grids], axis=1)
    best = np.full(len(coords), width + 1)
    ax = np.zeros(len(coords), dtype=np.int64)
    sg = np.zeros(len(coords), dtype=np.int64)
    for a in range(ndim):
        dl = coords[:, a]
        dr = shape[a] - 1 - coords[:, a]
        if not (a == 1 and freetop):
            m = dl < best
            best = np.where(m, dl, best)
            ax = np.where(m, a, ax)
            sg = np.where(m, -1, sg)
        m = dr < best
        best = np.where(m, dr, best)
        ax = np.where(m, a, ax)
        sg = np.where(m, 1, sg)
    keep = best <= width
    return coords[keep], ax[keep], sg[keep]


def gather_index(shape, coords, ax, sg):
    """For every layer node, the column-major flat indices of its 3^d block
    in the kernel's order (outward normal u, then the transverse axes in
    increasing order), -1 where the node is not interior."""
    ndim = len(shape)
    others = {a: [b for b in range(ndim) if b != a] for a in range(ndim)}
    t1 = np.array([others[a][0] for a in ax], dtype=np.int64)
    t2 = np.array([others[a][1] if ndim == 3 else 0 for a in ax], dtype=np.int64)
    rows = np.arange(len(coords))
    idx = []
    for u in (-1, 0, 1):
        for v in (-1, 0, 1):
            for w in ((-1, 0, 1) if ndim == 3 else (0,)):
                d = np.zeros((len(coords), ndim), dtype=np.int64)
                d[rows, ax] = sg * u
                d[rows, t1] = v
                if ndim == 3:
                    d[rows, t2] = w
                c = coords + d
                inside = np.ones(len(coords), dtype=bool)
                for a in range(ndim):
                    inside &= (c[:, a] >= 1) & (c[:, a] <= shape[a] - 2)
                flat = c[:, 0] + shape[0] * c[:, 1]
                if ndim == 3:
                    flat = flat + shape[0] * shape[1] * c[:, 2]
                idx.append(np.where(inside, flat, -1))
    return np.stack(idx, axis=1)


def gather(fields, gidx):
    """Inputs (n_nodes, 3 * 3^d) from three fields (time levels t-2, t-1, t)
    given in column-major order, and the flat index of each node's block."""
    out = []
    for f in fields:
        flat = np.ravel(f, order="F")
        g = np.where(gidx >= 0, flat[np.maximum(gidx, 0)], 0.0)
        out.append(g)
    return np.concatenate(out, axis=1)


# ---- training ---------------------------------------------------------------

def _pad_model(vel, pad, halo, freetop):
    """The model padded by `pad` + `halo` nodes on every absorbing side by
    repeating its edge values; returns (padded, offset of the original)."""
    ndim = vel.ndim
    widths = []
    off = []
    for a in range(ndim):
        left = 0 if (a == 1 and freetop) else pad + halo
        widths.append((left, pad + halo))
        off.append(left)
    return np.asfortranarray(np.pad(vel, widths, mode="edge")), off


def reference_fields(pkg, lengths, vel, srcs, recs, *, dt, nt, width, pad=300, halo=20,
                     freetop=True, ctx=None):
    """Fields of a reflection-free reference run on the small grid of `vel`
    (the model padded by pad + a CPML band of `halo`), FP64, one per step:
    yields (t, p_{t+1} restricted to the small grid). Positions in metres
    refer to the small grid."""
    ctx = ctx or default_context()
    big, off = _pad_model(vel, pad, halo, freetop)
    d = [lengths[a] / (vel.shape[a] - 1) for a in range(vel.ndim)]
    shift = np.array([off[a] * d[a] for a in range(vel.ndim)])
    Lb = [(big.shape[a] - 1) * d[a] for a in range(vel.ndim)]
    S = pkg.Sources(np.asarray(srcs.positions) + shift, srcs.t0s, srcs.srctfs, srcs.freqdomain)
    R = pkg.Receivers(np.asarray(recs.positions) + shift)
    s = prepare(Lb, None, big, S, R, halo=halo, rcoef=1e-4, ppw=1e-9, freetop=freetop,
                precision="f64", dt=dt, nt=nt)
    plan = ctx.plan(s["problem"], s["vel"], s["coeffs"], s["possrcs"], s["dt2srctf"],
                    s["posrecs"])
    sl = tuple(slice(off[a], off[a] + vel.shape[a]) for a in range(vel.ndim))
    try:
        for t in range(nt):
            plan.run(1, graph=False)
            yield t, np.asfortranarray(plan.field()[sl])
    finally:
        plan.close()


def training_data(pkg, cases, *, width=4, pad=300, every=1, keep=1.0, seed=0, ctx=None):
    """Inputs (the 3^d block at three levels normalised by its largest
    magnitude, then the Courant number) and targets (normalised alike) from
    the reference runs of `cases`: dicts with lengths, vel, srcs, recs, dt, nt,
    freetop. Samples whose inputs are all zero are dropped."""
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for c in cases:
        shape = c["vel"].shape
        coords, ax, sg = layer_nodes(shape, width, c["freetop"])
        gidx = gather_index(shape, coords, ax, sg)
        flat_node = coords[:, 0] + shape[0] * coords[:, 1]
        if len(shape) == 3:
            flat_node = flat_node + shape[0] * shape[1] * coords[:, 2]
        d = [c["lengths"][a] / (shape[a] - 1) for a in range(len(shape))]
        r = courant(c["vel"], c["dt"], d, coords, ax)
        hist = [np.zeros(shape, order="F")] * 3  # p_{t-2}, p_{t-1}, p_t
        for t, pnew in reference_fields(pkg, c["lengths"], c["vel"], c["srcs"], c["recs"],
                                        dt=c["dt"], nt=c["nt"], width=width, pad=pad,
                                        freetop=c["freetop"], ctx=ctx):
            if t % every == 0:
                x = gather(hist, gidx)
                y = np.ravel(pnew, order="F")[flat_node]
                s = np.abs(x).max(axis=1)
                m = s > 0
                if keep < 1.0:
                    m &= rng.random(len(m)) < keep
                X.append(np.concatenate([x[m] / s[m, None], r[m, None]], axis=1).astype(np.float32))
                Y.append((y[m] / s[m]).astype(np.float32))
            hist = [hist[1], hist[2], pnew]
    return np.concatenate(X), np.concatenate(Y)


def train(X, Y, *, epochs=8, batch=8192, lr=2e-3, seed=0, noise=0.0, device="cuda", log=None):
    """Fits K -> 32 -> 32 -> 1 (ReLU) by mean squared error with Adam (inputs
    perturbed by Gaussian noise of std `noise`, which makes the layer less
    sensitive to its own errors when it runs step after step); returns the
    weights as a flat float32 array (pack() order), rounded to BF16."""
    import torch
    torch.manual_seed(seed)
    k = X.shape[1]
    net = torch.nn.Sequential(torch.nn.Linear(k, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, 1)).to(device)
    Xt = torch.from_numpy(X).to(device)
    Yt = torch.from_numpy(Y).to(device)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=epochs)
    n = Xt.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n, device=device)
        tot = 0.0
        for b in range(0, n, batch):
            sel = perm[b:b + batch]
            xb = Xt[sel]
            if noise > 0:
                xb = xb + noise * torch.randn_like(xb)
            loss = torch.mean((net(xb).squeeze(1) - Yt[sel]) ** 2)
            opt.zero_grad()
            loss.backward()
            opt.step()
            tot += float(loss.detach()) * len(sel)
        sched.step()
        if log:
            log(f"epoch {ep}: mse {tot / n:.3e}")
    l1, l2, l3 = net[0], net[2], net[4]
    flat = pack(l1.weight.detach().cpu().numpy(), l1.bias.detach().cpu().numpy(),
                l2.weight.detach().cpu().numpy(), l2.bias.detach().cpu().numpy(),
                l3.weight.detach().cpu().numpy().ravel(), float(l3.bias.detach().cpu()))
    return from_bf16(to_bf16(flat))


class RolloutSim:
    """The learned-layer step of one 2D case as torch operations (the
    kernel's scheme, differentiable), for training through the time loop.
    Fields are (ny, nx) tensors, so that flat index i + nx j matches the
    kernel's column-major order."""

    def __init__(self, vel, dt, d, width, freetop, src_node, stf, device="cuda"):
        import torch
        nx, ny = vel.shape
        self.nx, self.ny = nx, ny
        self.F = torch.tensor((dt * dt * vel.astype(np.float64) ** 2).T, dtype=torch.float32,
                              device=device)
        self.inv2 = [1.0 / (d[0] * d[0]), 1.0 / (d[1] * d[1])]
        coords, ax, sg = layer_nodes((nx, ny), width, freetop)
        gidx = gather_index((nx, ny), coords, ax, sg)
        self.lflat = torch.tensor(coords[:, 0] + nx * coords[:, 1], device=device)
        self.gidx = torch.tensor(np.maximum(gidx, 0), device=device)
        self.gmask = torch.tensor(gidx >= 0, device=device, dtype=torch.float32)
        self.r = torch.tensor(courant(vel, dt, d, coords, ax), dtype=torch.float32,
                              device=device)[:, None]
        core = np.zeros((ny, nx), dtype=bool)
        core[1:ny - 1, 1:nx - 1] = True
        lm = np.zeros(nx * ny, dtype=bool)
        lm[coords[:, 0] + nx * coords[:, 1]] = True
        core &= ~lm.reshape(ny, nx)
        self.core = torch.tensor(core, device=device, dtype=torch.float32)
        self.src = int(src_node[0] + nx * src_node[1])
        self.stf = torch.tensor(stf, dtype=torch.float32, device=device)

    def step(self, net, p0, p1, p2, t):
        import torch
        lap = torch.zeros_like(p2)
        c = p2[1:-1, 1:-1]
        lap[1:-1, 1:-1] = ((p2[1:-1, 2:] - 2 * c + p2[1:-1, :-2]) * self.inv2[0] +
                           (p2[2:, 1:-1] - 2 * c + p2[:-2, 1:-1]) * self.inv2[1])
        new = (2 * p2 - p1 + self.F * lap) * self.core
        x = torch.cat([f.reshape(-1)[self.gidx] * self.gmask for f in (p0, p1, p2)], dim=1)
        sc = torch.amax(x.abs(), dim=1).clamp_min(1e-30)
        y = net(torch.cat([x / sc[:, None], self.r], dim=1)).squeeze(1) * sc
        new = new.reshape(-1).index_put((self.lflat,), y, accumulate=True).reshape(p2.shape)
        if t < self.stf.shape[0]:
            new = new.reshape(-1).index_put((torch.tensor([self.src], device=new.device),),
                                            self.stf[t:t + 1], accumulate=True).reshape(p2.shape)
        return new


def train_rollout(net_flat, sims, refs, *, window=100, iters=400, lr=5e-4, seed=0,
                  device="cuda", log=None):
    """Fine-tunes MLP weights (pack() order) through `window` steps of the
    learned-layer scheme: each iteration starts from a reference state of a
    random case and time and penalises the squared difference to the
    reference fields over the window, relative to their energy. sims:
    RolloutSim per case; refs: (nt, ny, nx) reference fields per case."""
    import torch
    rng = np.random.default_rng(seed)
    k = sims[0].gidx.shape[1] * 3 + 1
    W1, b1, W2, b2, W3, b3 = unpack(net_flat, 2)
    net = torch.nn.Sequential(torch.nn.Linear(k, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, 1)).to(device)
    with torch.no_grad():
        for lin, (w, b) in zip((net[0], net[2], net[4]), ((W1, b1), (W2, b2), (W3[None, :], [b3]))):
            lin.weight.copy_(torch.tensor(np.asarray(w), dtype=torch.float32))
            lin.bias.copy_(torch.tensor(np.asarray(b, dtype=np.float32)))
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    for itn in range(iters):
        c = int(rng.integers(len(sims)))
        sim, ref = sims[c], refs[c]
        nt = ref.shape[0]
        t0 = int(rng.integers(3, nt - window))
        p0, p1, p2 = ref[t0 - 3], ref[t0 - 2], ref[t0 - 1]
        loss = 0.0
        norm = 0.0
        for t in range(t0, t0 + window):
            new = sim.step(net, p0, p1, p2, t - 1)
            r = ref[t]
            loss = loss + torch.sum((new - r) ** 2)
            norm = norm + torch.sum(r ** 2)
            p0, p1, p2 = p1, p2, new
        loss = loss / norm.clamp_min(1e-30)
        opt.zero_grad()
        loss.backward()
        torch.nn.utils.clip_grad_norm_(net.parameters(), 1.0)
        opt.step()
        if log and itn % 50 == 0:
            log(f"rollout iter {itn}: relative error {float(loss.detach()):.3e}")
    l1, l2, l3 = net[0], net[2], net[4]
    flat = pack(l1.weight.detach().cpu().numpy(), l1.bias.detach().cpu().numpy(),
                l2.weight.detach().cpu().numpy(), l2.bias.detach().cpu().numpy(),
                l3.weight.detach().cpu().numpy().ravel(), float(l3.bias.detach().cpu()))
    return from_bf16(to_bf16(flat))


def fit_linear(X, Y, ridge=1e-6):
    """Least-squares linear layer y = a·x (ridge-regularised), written as MLP
    weights: two hidden units carry +a·x and -a·x through the ReLUs."""
    k = X.shape[1]
    A = X.astype(np.float64)
    G = A.T @ A + ridge * len(A) * np.eye(k)
    a = np.linalg.solve(G, A.T @ Y.astype(np.float64))
    W1 = np.zeros((HIDDEN, k))
    W1[0], W1[1] = a, -a
    W2 = np.zeros((HIDDEN, HIDDEN))
    W2[0, 0] = W2[1, 1] = 1.0
    W3 = np.zeros(HIDDEN)
    W3[0], W3[1] = 1.0, -1.0
    return pack(W1, np.zeros(HIDDEN), W2, np.zeros(HIDDEN), W3, 0.0)


def damped(flat, gamma, ndim):
    """Weights whose output is scaled by (1 - gamma)."""
    W1, b1, W2, b2, W3, b3 = unpack(flat, ndim)
    return pack(W1, b1, W2, b2, W3 * (1.0 - gamma), b3 * (1.0 - gamma))


def reflected_energy(traces, reference):
    """Σ (traces - reference)² / Σ reference² over all samples."""
    return float(np.sum((traces - reference) ** 2) / max(np.sum(reference ** 2), 1e-300))
