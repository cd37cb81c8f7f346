"""The exchange hook of a shot-sharded run, on one GPU.

Two contexts hold the two shards of a survey.  They run one after the other (never two
kernels that wait on each other): the first with a hook that records what it would send,
the second with a hook that adds the first's record -- which is what a two-rank all-reduce
hands the second rank.  The second context's gradient and misfit must then be the whole
survey's.  The NCCL hook itself (fwiedu.dist.device_hook) runs on a one-rank NCCL process
group through a whole FWI iteration, where the sum over one rank must change nothing.
"""
import os
import socket

import numpy as np
import pytest

from fwiedu import dist as D
from fwiedu import engine as E
from golden_cases import Case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _ctx(c, shots, obs):
    ctx = E.Context(0)
    ctx.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    ctx.set_shots(shots)
    ctx.set_observed(obs)
    return ctx


def _view(ptr, count):
    import torch
    return torch.as_tensor(D._DeviceDoubles(ptr, count), device="cuda:0")


def test_two_shards_sum_to_the_whole_survey():
    import torch
    c = Case("fs1_small")
    full = _ctx(c, c.shots, c.obs)
    full.run(1, 10.0, 2, c.precondition, E.PATH_BATCHED)
    g_full, f_full = full.gradient(), full.objective()
    full.close()

    parts = [D.shard(c.shots, 2, r) for r in range(2)]
    sent = []

    def record(ptr, count, stream):
        torch.cuda.ExternalStream(stream).synchronize()
        sent.append(_view(ptr, count).clone())

    def add_record(ptr, count, stream):
        k = add_record.calls
        add_record.calls += 1
        torch.cuda.ExternalStream(stream).synchronize()
        t = _view(ptr, count)
        t += sent[k]
        torch.cuda.synchronize()

    add_record.calls = 0
    a = _ctx(c, [c.shots[i] for i in parts[1]], [c.obs[i] for i in parts[1]])
    a.set_allreduce(record)
    a.run(1, 10.0, 2, c.precondition, E.PATH_BATCHED)
    a.objective()
    a.close()
    assert len(sent) == 2 and sent[0].numel() == 2 * c.vp0.size and sent[1].numel() == 1

    b = _ctx(c, [c.shots[i] for i in parts[0]], [c.obs[i] for i in parts[0]])
    b.set_allreduce(add_record)
    b.run(1, 10.0, 2, c.precondition, E.PATH_BATCHED)
    g, f = b.gradient(), b.objective()
    b.close()
    assert add_record.calls == 2
    assert rel(g, g_full) <= 1e-6 and rel(g, c.grad) <= 1e-6
    assert abs(f - f_full) <= 1e-12 * abs(f_full)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_hook_one_rank_changes_nothing():
    import torch.distributed as dist
    c = Case("fs1_small")
    P = dict(rx=2, rz=1, precondition=1, filter=2, freq=10.0, waterdepth=6, vp_water=1500.0, rho_water=1000.0,
             vpmin=1500.0, vpmax=4700.0, rhomin=1000.0, rhomax=2700.0, gardner=1)
    ref = _ctx(c, c.shots, c.obs)
    r0 = ref.fwi_iteration(E.IterParams(path=E.PATH_BATCHED, **P))
    m0 = ref.model()
    ref.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        ctx = _ctx(c, c.shots, c.obs)
        ctx.set_allreduce(D.device_hook(0))
        r1 = ctx.fwi_iteration(E.IterParams(path=E.PATH_BATCHED, **P))
        m1 = ctx.model()
        ctx.close()
    finally:
        dist.destroy_process_group()
    for k in ("fun1", "fun2", "steplen", "scalar"):
        assert r0[k] == r1[k], k
    assert np.array_equal(m0[0], m1[0]) and np.array_equal(m0[1], m1[1])
