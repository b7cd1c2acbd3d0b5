"""numpy FP64 restatement of the learned thin-layer solve (test
infrastructure only): the scheme of awc_forward_learned
(acousticwavecpml.jl_b200/csrc/awc_learned.cu), written independently here
so that the GPU result can be checked against it. It has no counterpart in
the reference, whose absorbing boundary is the CPML.

Interior nodes: p_{t+1} = 2 p_t - p_{t-1} + F lap(p_t), F = dt² c². Layer
nodes (within `width` of an absorbing side): p_{t+1} = s MLP(x / s), x the
3^d block around the node at levels t-2, t-1, t (0 outside the interior),
ordered by level, then along the nearest side's outward normal (-1, 0, +1),
then along the remaining axes in increasing order; s = max |x| (1 when 0).
MLP: K -> 32 -> 32 -> 1 with ReLU over (x / s, r), r = sqrt(F) / d along
the normal (the local Courant number), K = 3 * 3^d + 1. Sources are added after the update, then
receivers sample p_{t+1}.
"""
import numpy as np


def _layer(shape, width, freetop):
    ndim = len(shape)
    out = []
    for idx in np.ndindex(*[n - 2 for n in shape]):
        c = [v + 1 for v in idx]
        best, ax, sg = width + 1, 0, 1
        for a in range(ndim):
            dl, dr = c[a], shape[a] - 1 - c[a]
            if not (a == 1 and freetop) and dl < best:
                best, ax, sg = dl, a, -1
            if dr < best:
                best, ax, sg = dr, a, 1
        if best <= width:
            out.append((tuple(c), ax, sg))
    return out


def _block(shape, c, ax, sg):
    ndim = len(shape)
    others = [b for b in range(ndim) if b != ax]
    pos = []
    for u in (-1, 0, 1):
        for v in (-1, 0, 1):
            for w in ((-1, 0, 1) if ndim == 3 else (0,)):
                d = [0] * ndim
                d[ax] = sg * u
                d[others[0]] = v
                if ndim == 3:
                    d[others[1]] = w
                q = tuple(c[a] + d[a] for a in range(ndim))
                inside = all(1 <= q[a] <= shape[a] - 2 for a in range(ndim))
                pos.append(q if inside else None)
    return pos


def forward(vel, d, dt, nt, width, freetop, weights, src_nodes, stf, rec_nodes):
    """vel (nx, ny[, nz]); d spacings; weights (W1, b1, W2, b2, W3, b3) as
    float arrays; src_nodes / rec_nodes lists of 0-based index tuples; stf
    (nt, nsrc) injected values. Returns (traces (nt, nrec), final field)."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(x, dtype=np.float64) for x in weights]
    shape = vel.shape
    ndim = vel.ndim
    F = dt * dt * vel.astype(np.float64) ** 2
    layer = _layer(shape, width, freetop)
    blocks = [_block(shape, c, ax, sg) for c, ax, sg in layer]
    is_layer = np.zeros(shape, dtype=bool)
    for c, _, _ in layer:
        is_layer[c] = True
    inner = tuple(slice(1, n - 1) for n in shape)
    hist = [np.zeros(shape) for _ in range(3)]  # p_{t-2}, p_{t-1}, p_t
    traces = np.zeros((nt, len(rec_nodes)))
    for t in range(nt):
        p0, p1, p2 = hist
        new = np.zeros(shape)
        lap = np.zeros(shape)
        for a in range(ndim):
            sl_c = list(inner)
            sl_p = list(inner)
            sl_m = list(inner)
            sl_p[a] = slice(2, shape[a])
            sl_m[a] = slice(0, shape[a] - 2)
            lap[inner] += (p2[tuple(sl_p)] - 2.0 * p2[inner] + p2[tuple(sl_m)]) / (d[a] * d[a])
        upd = 2.0 * p2 - p1 + F * lap
        new[inner] = upd[inner]
        for (c, ax, _), blk in zip(layer, blocks):
            x = np.array([lv[q] if q is not None else 0.0 for lv in (p0, p1, p2) for q in blk])
            s = np.abs(x).max()
            xs = x / s if s > 0 else x
            xs = np.append(xs, np.sqrt(np.float32(F[c])) / d[ax])
            h1 = np.maximum(W1 @ xs + b1, 0.0)
            h2 = np.maximum(W2 @ h1 + b2, 0.0)
            y = float(W3 @ h2 + b3)
            new[c] = y * (s if s > 0 else 1.0)
        for k, n in enumerate(src_nodes):
            new[n] += stf[t, k]
        for r, n in enumerate(rec_nodes):
            traces[t, r] = new[n]
        hist = [p1, p2, new]
    return traces, hist[2]
