"""Memory-bounded waves of the batched path.

When the frame blocks of a whole survey do not fit in device memory, fwi_ctx_run runs the shots
of each geometry group in waves through one reused frame pool.  FWI_WAVE caps the shots per wave
so that the schedule runs on a small survey: the traces, the gradient and the misfit must be the
single-wave run's bit for bit (the shots are independent and the stack runs once, after the last
wave), and runs alternating between the two schedules must not disturb each other.
"""
import os

import numpy as np
import pytest

from fwiedu import engine as E
from golden_cases import Case

pytestmark = pytest.mark.gpu


def _ctx(c):
    ctx = E.Context(0)
    ctx.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    ctx.set_shots(c.shots)
    ctx.set_observed(c.obs)
    return ctx


def _run(ctx, c, nshot, wave):
    if wave:
        os.environ["FWI_WAVE"] = str(wave)
    else:
        os.environ.pop("FWI_WAVE", None)
    try:
        ctx.run(0, path=E.PATH_BATCHED)
        traces = [ctx.traces(i) for i in range(nshot)]
        ctx.run(1, 10.0, int(c.filter), c.precondition, E.PATH_BATCHED)
        return traces, ctx.gradient(), ctx.objective()
    finally:
        os.environ.pop("FWI_WAVE", None)


@pytest.mark.parametrize("name", ["fs1_small", "filt0"])
def test_waves_match_one_wave(name):
    c = Case(name)
    n = len(c.shots)
    ctx = _ctx(c)
    try:
        t0, g0, f0 = _run(ctx, c, n, 0)
        for wave in (1, 2, 0, 1):  # back and forth between the schedules on one context
            t, g, f = _run(ctx, c, n, wave)
            assert all(np.array_equal(a, b) for a, b in zip(t, t0)), wave
            assert np.array_equal(g, g0), wave
            assert f == f0, wave
    finally:
        ctx.close()
    rel = np.linalg.norm(g0.astype(np.float64) - c.grad) / np.linalg.norm(c.grad)
    assert rel <= 1e-4  # and the single-wave gradient is the reference's (golden vectors)


def test_budget_below_the_survey_brings_waves():
    """A context whose budget holds the shots' own buffers but not every frame block runs the
    gradient in waves by itself, within its budget, with the unbounded run's results."""
    c = Case("fs1_small")
    n = len(c.shots)
    ref = _ctx(c)
    try:
        ref.run(1, 10.0, int(c.filter), c.precondition, E.PATH_BATCHED)
        g0, f0, held0 = ref.gradient(), ref.objective(), ref.stats()["device_bytes"]
    finally:
        ref.close()
    one = E.Context(0)  # the footprint of a one-shot run of the same model
    try:
        one.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
        one.set_shots(c.shots[:1])
        one.set_observed(c.obs[:1])
        one.run(1, 10.0, int(c.filter), c.precondition, E.PATH_BATCHED)
        held1 = one.stats()["device_bytes"]
    finally:
        one.close()
    budget = held1 + (held0 - held1) // 2  # about half of the other shots' state
    ctx = E.Context(0, budget)
    try:
        ctx.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
        ctx.set_shots(c.shots)
        ctx.set_observed(c.obs)
        ctx.run(1, 10.0, int(c.filter), c.precondition, E.PATH_BATCHED)
        g, f, held = ctx.gradient(), ctx.objective(), ctx.stats()["device_bytes"]
    finally:
        ctx.close()
    assert n >= 3 and held <= budget < held0
    assert np.array_equal(g, g0) and f == f0
