"""Multi-process host logic on CPU (gloo, world size 2): shots are split
rank, rank + N, ... and the gradient and misfit are summed with one
all-reduce, so every rank ends with the same total as a single process."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shot_gradient(shot):
    """A deterministic stand-in for one shot's (misfit, dJ/dc²)."""
    rng = np.random.default_rng(shot)
    return float(shot) + 0.5, rng.standard_normal((7, 5, 3))


def _worker(rank, world, port, shots, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import __graft_entry__ as g
    pkg = g.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        J, grad = pkg.adjoint.sharded_gradient(shots, _shot_gradient, (7, 5, 3))
        mine = shots[rank::world]
        np.save(os.path.join(out, f"r{rank}.npy"), np.concatenate([[J, len(mine)], grad.ravel()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nshots", [5, 1])
def test_sharded_gradient_gloo(tmp_path, nshots):
    import torch.multiprocessing as mp
    shots = list(range(nshots))
    mp.spawn(_worker, args=(2, _free_port(), shots, str(tmp_path)), nprocs=2, join=True)
    J_ref = sum(_shot_gradient(s)[0] for s in shots)
    g_ref = sum(_shot_gradient(s)[1] for s in shots)
    counts = 0
    for r in range(2):
        a = np.load(tmp_path / f"r{r}.npy")
        assert abs(a[0] - J_ref) <= 1e-12 * J_ref
        counts += int(a[1])
        np.testing.assert_allclose(a[2:].reshape(7, 5, 3), g_ref, rtol=1e-12, atol=1e-12)
    assert counts == nshots  # every shot on exactly one rank


def test_sharded_gradient_single_process():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as g
    pkg = g.load_package()
    J, grad = pkg.adjoint.sharded_gradient([3, 4], _shot_gradient, (7, 5, 3))
    assert J == 3.5 + 4.5
    np.testing.assert_allclose(grad, _shot_gradient(3)[1] + _shot_gradient(4)[1])
