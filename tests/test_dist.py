"""Shot sharding and the one exchange step of a sharded gradient, on CPU.

The partition (fwiedu.dist.shard) is checked directly.  The exchange is checked end to end
with two gloo ranks: each rank computes the per-shot gradients and pseudo-Hessians of its
shots with the oracle, stacks them in FP64, sums the stacks over the ranks with
fwiedu.dist.allreduce_ (the same call the NCCL device hook makes), applies the global
preconditioning and must land on the single-process gradient of the whole survey --
the golden gradient of the reference.
"""
import os
import socket
import sys

import numpy as np
import pytest

from fwiedu import dist as D
from fwiedu.models import Shot

HERE = os.path.dirname(os.path.abspath(__file__))


def fake_shots(widths, ns):
    return [Shot(shotID=i, isx=0, isz=1, igx=np.zeros(1, np.int32), igz=np.zeros(1, np.int32), ns=n, sampleRate=1,
                 ix_min=0, ix_max=w - 1, dt=0.001, dtr=10.0, fpeak=10.0, src=np.zeros(n, np.float32), sx=0.0, sz=0.0)
            for i, (w, n) in enumerate(zip(widths, ns))]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_is_a_partition(world):
    shots = fake_shots([100 + 7 * (i % 5) for i in range(23)], [300 + 50 * (i % 3) for i in range(23)])
    parts = [D.shard(shots, world, r) for r in range(world)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(shots)))
    assert all(p == sorted(p) for p in parts)  # survey order inside a rank
    assert all(len(p) >= 1 for p in parts)
    loads = [sum(D.shot_cost(shots[i]) for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(D.shot_cost(s) for s in shots)
    assert parts == [D.shard(shots, world, r) for r in range(world)]  # deterministic


def test_equal_shots_go_round_robin():
    shots = fake_shots([601] * 60, [4001] * 60)
    assert D.shard(shots, 4, 1) == list(range(1, 60, 4))


def test_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        D.shard(fake_shots([10], [10]), 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path[:0] = [os.path.join(HERE, "..", "fwi-edu_b200"), os.path.join(HERE, "..", "oracle"), HERE]
    import torch
    import torch.distributed as dist

    import pyoracle
    from fwiedu import dist as DD
    from golden_cases import Case

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = Case("fs1_small")
        port32 = pyoracle.Port(32)
        nx, nz = c.vp0.shape
        gc = np.zeros((nx, nz), np.float64)
        hc = np.zeros((nx, nz), np.float64)
        for i in DD.shard(c.shots, world, rank):
            s = c.shots[i]
            _, g, h = port32.shot_gradient(s, c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 10.0, 2,
                                           c.precondition, c.obs[i])
            gc[s.ix_min:s.ix_max + 1] += g
            hc[s.ix_min:s.ix_max + 1] += h
        stacks = torch.from_numpy(np.stack([gc, hc]))
        DD.allreduce_(stacks)
        grad = stacks[0].numpy().astype(np.float32)
        prec = stacks[1].numpy().astype(np.float32)
        if c.precondition == 1:
            port32.global_precondition(grad, prec)
        np.save(os.path.join(out, f"grad{rank}.npy"), grad)
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_gloo_matches_reference(tmp_path):
    import torch.multiprocessing as mp

    from golden_cases import Case

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    c = Case("fs1_small")
    g0 = np.load(tmp_path / "grad0.npy")
    g1 = np.load(tmp_path / "grad1.npy")
    assert np.array_equal(g0, g1)  # every rank holds the same gradient after the exchange
    rel = np.linalg.norm(g0.astype(np.float64) - c.grad) / np.linalg.norm(c.grad)
    assert rel <= 1e-6  # FP64 partial sums in another order than the reference's shot loop
