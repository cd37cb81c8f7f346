"""Continuous batching (fwi_exec_*): runs of different contexts -- different grid sizes, record
lengths, problems and shot counts -- advanced by the same step launches, each joining the batch
while the others are in flight.  Every run must give the bits it gives alone on the batched path
of fwi_ctx_run (and so the reference's golden vectors where it is a golden case)."""
import numpy as np
import pytest

from fwiedu import engine as E
from fwiedu import models as M
from golden_cases import Case

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _survey(nz, nx, nt, dx, dt, nshot, seed, f=10.0):
    vp = M.layered_model(nz, nx, seed=seed, water_rows=6, anom_sigma=4)
    src = M.ricker(nt, dt, f, 1.5 / f)
    sv = M.line_survey(nz, nx, dx, dx, dt, nt, nshot, src, spacing_cells=max(1, (nx - 10) // nshot), first_cell=5)
    return vp, M.gardner(vp, water_rows=6), M.survey_shots(sv)


def _jobs():
    """(model args, shots, problem, observed or None) of four runs"""
    c = Case("fs1_small")
    vp1, rho1, sh1 = _survey(221, 601, 700, 12.5, 0.001, 5, seed=21)
    vp2, rho2, sh2 = _survey(90, 300, 500, 10.0, 0.001, 3, seed=22, f=15.0)
    obs2 = [np.zeros((len(s.igx), s.ns), np.float32) for s in sh2]
    obs2[0][:, 100:] = 1e-3  # a non-zero residual
    return [
        ((c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs), c.shots, 1, c.obs),
        ((vp1, rho1, 12.5, 12.5, 0.001, 700, 40, 1), sh1, 0, None),
        ((vp2, rho2, 10.0, 10.0, 0.001, 500, 20, 0), sh2, 1, obs2),
        ((c.vp1, c.rho1, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs), c.shots, 2, c.obs),
    ]


def _ctx(model, shots, obs):
    ctx = E.Context(0)
    ctx.set_model(*model)
    ctx.set_shots(shots)
    if obs is not None:
        ctx.set_observed(obs)
    return ctx


def _results(ctx, problem, n):
    tr = [ctx.traces(i) for i in range(n)]
    return tr, (ctx.gradient() if problem == 1 else None)


def test_runs_joining_a_batch_match_their_runs_alone():
    jobs = _jobs()
    alone = []
    for model, shots, problem, obs in jobs:
        ctx = _ctx(model, shots, obs)
        ctx.run(problem, 10.0, 2, 1, E.PATH_BATCHED)
        alone.append(_results(ctx, problem, len(shots)))
        ctx.close()
    ex = E.Executor(0)
    ctxs = [_ctx(m, s, o) for m, s, _, o in jobs]
    try:
        ex.add(ctxs[0], jobs[0][2], 10.0, 2, 1)
        ex.step(57)                      # the first run is mid-way through its forward pass
        ex.add(ctxs[1], jobs[1][2], 10.0, 2, 1)
        ex.add(ctxs[2], jobs[2][2], 10.0, 2, 1)
        ex.step(333)
        ex.add(ctxs[3], jobs[3][2], 10.0, 2, 1)
        assert ex.step(0) == 0
        assert ex.launches() < sum(1 + 2 * m[5] for m, *_ in jobs)  # the runs shared launches
        for k, (ctx, (model, shots, problem, obs)) in enumerate(zip(ctxs, jobs)):
            done, status = ex.poll(ctx)
            assert done and status == 0, (k, status)
            tr, g = _results(ctx, problem, len(shots))
            for i in range(len(shots)):
                assert np.array_equal(tr[i], alone[k][0][i]), (k, i)
            if problem == 1:
                assert np.array_equal(g, alone[k][1]), k
    finally:
        ex.close()
        for c in ctxs:
            c.close()
    # the golden cases against the reference's own outputs
    c = Case("fs1_small")
    assert rel(alone[0][1], c.grad) <= 1e-6
    for i in range(c.nshot):
        assert np.array_equal(alone[0][0][i], c.adj[i])
        assert np.array_equal(alone[3][0][i], c.res[i])
