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


# ---- the real sharding code with the oracle standing in for the device -----
# Small 2D shots (the shape of the batched workload: surface sources, one
# model per shot family); each rank runs the oracle on its shard.

def _oracle_shots():
    rng = np.random.default_rng(17)
    shots = []
    for k in range(5):
        nx, ny, d = 41 + 4 * k, 31, 10.0
        vel = 2000.0 + 10.0 * np.arange(ny)[None, :] + 50.0 * rng.random((nx, ny))
        shots.append(dict(lengths=((nx - 1) * d, (ny - 1) * d), vel=np.asfortranarray(vel),
                          src=[[(5 + 3 * k) * d, 2 * d]], rec=[[(i - 1) * d, 2 * d]
                                                                for i in range(3, nx - 2, 4)],
                          f0=15.0, nt=120))
    return shots


def _oracle_traces(shot):
    sys.path.insert(0, ROOT)
    import __graft_entry__ as g
    O = g.load_oracle()
    so = O.setup(shot["lengths"], None, shot["vel"], shot["src"], [0.05], shot["f0"],
                 shot["rec"], halo=6, rcoef=1e-4, freetop=True, nt=shot["nt"], check_ppw=False)
    pend, tr = O.forward(so, nthreads=1)
    return pend, tr


def _oracle_shot_gradient(shot):
    """(misfit against zero data, a field-shaped array) of one shot, both from
    the oracle's arithmetic; stands in for awc_misfit_gradient on CPU."""
    pend, tr = _oracle_traces(shot)
    return 0.5 * float(np.sum(tr ** 2)), pend[:41, :]


def _real_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import __graft_entry__ as g
    pkg = g.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shots = _oracle_shots()
        ran = []

        def run(mine):
            ran.extend(s["src"][0][0] for s in mine)
            return [_oracle_traces(s)[1] for s in mine]

        traces = pkg.solve_sharded(shots, run)
        J, grad = pkg.adjoint.sharded_gradient(shots, _oracle_shot_gradient, (41, 31))
        batches = []

        def batch(mine):
            # the rank's shots in one call, summed in order (as
            # misfit_gradient_shots does on the device)
            batches.append([s["src"][0][0] for s in mine])
            Jb, gb = 0.0, np.zeros((41, 31), order="F")
            for s in mine:
                j, g = _oracle_shot_gradient(s)
                Jb += j
                gb += g
            return Jb, gb

        Jb, gradb = pkg.adjoint.sharded_gradient(shots, batch, (41, 31), batched=True)
        np.savez(os.path.join(out, f"r{rank}.npz"), J=J, grad=grad, ran=np.array(ran),
                 Jb=Jb, gradb=gradb, batches=np.array(batches),
                 **{f"t{k}": t for k, t in enumerate(traces)})
    finally:
        dist.destroy_process_group()


def test_sharded_shots_and_gradient_with_oracle_gloo(tmp_path):
    """Two gloo ranks run the package's shot sharding (batch.shard via
    solve_sharded: rank r takes shots r, r + 2, ...; results gathered in shot
    order) and sharded_gradient (one all-reduce of [gradient, misfit]) with
    per-shot functions that run the oracle, per shot and batched (one call per
    rank with its shots). Both ranks must end with what a single process
    computes for the whole set."""
    import torch.multiprocessing as mp
    mp.spawn(_real_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    shots = _oracle_shots()
    ref_tr = [_oracle_traces(s)[1] for s in shots]
    J_ref, g_ref = 0.0, np.zeros((41, 31))
    for s in shots:
        j, g = _oracle_shot_gradient(s)
        J_ref += j
        g_ref += g
    ran = []
    for r in range(2):
        d = np.load(tmp_path / f"r{r}.npz")
        for k, t in enumerate(ref_tr):
            np.testing.assert_array_equal(d[f"t{k}"], t)
        for J, g in ((d["J"], d["grad"]), (d["Jb"], d["gradb"])):
            assert abs(float(J) - J_ref) <= 1e-12 * J_ref
            np.testing.assert_allclose(g, g_ref, rtol=1e-12, atol=1e-30)
        # one batched call per rank, with the rank's shots in order
        assert d["batches"].shape[0] == 1
        assert list(d["batches"][0]) == [s["src"][0][0] for s in shots[r::2]]
        ran += list(d["ran"])
    # each shot ran on exactly one rank
    assert sorted(ran) == sorted(s["src"][0][0] for s in shots)
