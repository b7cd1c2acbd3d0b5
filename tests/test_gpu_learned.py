"""The learned thin layer (awc_forward_learned) against the numpy FP64
restatement in oracle/learned_oracle.py: relative L2 <= 1e-4 on traces and
field (FP32 GPU against FP64), 2D and 3D, free top on and off, layer widths
1, 2, 4 and 8, with random BF16 weights (the solve must reproduce the scheme
for any weights) and with the shipped trained weights in 2D."""
import os
import sys

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import learned_oracle
    return learned_oracle


def _random_weights(L, ndim, rng):
    k = L.n_inputs(ndim)
    flat = L.pack(rng.standard_normal((32, k)) / np.sqrt(k), 0.05 * rng.standard_normal(32),
                  rng.standard_normal((32, 32)) / np.sqrt(32), 0.05 * rng.standard_normal(32),
                  rng.standard_normal(32) / np.sqrt(32) * 0.3, 0.01)
    return L.to_bf16(flat)


@pytest.mark.parametrize("ndim,freetop,trained,width", [
    (2, True, False, 4), (2, False, False, 4), (3, True, False, 4), (2, True, True, 4),
    (3, False, False, 2),   # every side absorbing, a thin layer
    (2, False, False, 1),   # one node: every block reaches the rim
    (2, True, False, 8),    # the widest layer
])
def test_learned_layer_vs_oracle(pkg, ctx, ndim, freetop, trained, width):
    from acousticwavecpml_b200 import learned as L
    rng = np.random.default_rng(ndim * 10 + freetop)
    shape = (36, 30) if ndim == 2 else (20, 18, 16)
    d = 10.0
    vel = 2000.0 + 300.0 * rng.random(shape)
    lengths = tuple((n - 1) * d for n in shape)
    src = [[(n // 2) * d for n in shape]]
    src[0][1] = 8 * d
    recs = [[3 * d, 5 * d] + ([6 * d] if ndim == 3 else []),
            [(shape[0] - 6) * d, 10 * d] + ([8 * d] if ndim == 3 else []),
            [(shape[0] // 2) * d, (shape[1] - 2) * d] + ([4 * d] if ndim == 3 else [])]
    S = pkg.Sources(src, [0.04], [pkg.rickersource1D], 20.0)
    R = pkg.Receivers(recs)
    nt = 120 if ndim == 2 else 80
    s = pkg.prepare(lengths, None, vel, S, R, halo=width, ppw=1e-9, freetop=freetop,
                    precision="f32", nt=nt)
    wb = L.load_weights() if trained else _random_weights(L, ndim, rng)
    tr, pf = L.forward_learned(s, wb, ctx)
    o = _oracle()
    nodes = lambda pos: [tuple(int(v) - 1 for v in row) for row in pos]
    tr_o, pf_o = o.forward(s["vel"], s["d"], s["dt"], nt, width, freetop,
                           L.unpack(L.from_bf16(wb), ndim), nodes(s["possrcs"]),
                           s["dt2srctf"], nodes(s["posrecs"]))
    e_t = cases.rel_l2(tr, tr_o)
    e_p = cases.rel_l2(pf, pf_o)
    print(f"learned {ndim}D freetop={freetop} trained={trained} width={width}: "
          f"traces {e_t:.2e} field {e_p:.2e}")
    assert np.abs(tr_o).max() > 0
    assert e_t <= 1e-4 and e_p <= 1e-4
