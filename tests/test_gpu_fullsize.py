"""Parity at the benchmarked size: two shots of the 60-shot 221 x 601 survey (nt = 4001,
40-cell absorbing layer, free surface, pseudo-Hessian preconditioning, filter 2).

This is the configuration the throughput figures are earned on: checkpoint interval
d = 89 with 45 stored pairs, 3912 replayed steps per shot, sources one row below the
free surface (the replay-order trap of propagation.c:558-564 vs :656-662 at its
sharpest) and a receiver in every column.  The oracle's FP32 restatement (bit-exact
against the reference's golden vectors) runs the same two shots; where the reference
itself was built (oracle/_ref/libfwiref_strict.so, its strict-IEEE build) the gradient
is checked against it directly as well.

Compared, on both engine paths (one shot per launch and the batched launch):
seismograms, adjoint sources (propagation.c:876-935), the stacked and preconditioned
gradient (:945-1011), the line-search residuals of a trial model (problem 2), and one
whole FWI iteration (acoustic2d_fwi.c:411-465) composed step by step from the oracle.
The contracted-FMA arithmetic (FWI_MATH=1) is held to the FP32 tolerance instead:
seismograms rel-L2 <= 1e-5, adjoint sources and gradient <= 1e-4.
"""
import os

import numpy as np
import pytest

from fwiedu import engine as E
from fwiedu import models as M

pytestmark = pytest.mark.gpu

NZ, NX, DX, DT, NT, PML, FS, WATER = 221, 601, 12.5, 0.001, 4001, 40, 1, 20
ITER = dict(rx=1, rz=1, precondition=1, filter=2, freq=10.0, waterdepth=WATER, vp_water=1500.0, rho_water=1000.0,
            vpmin=1500.0, vpmax=4700.0, rhomin=1000.0, rhomax=2700.0, gardner=1)
KEYS = ("FWI_TX", "FWI_NST", "FWI_CHUNK", "FWI_KERNEL", "FWI_MATH", "FWI_TUNE", "FWI_GPT", "FWI_OCC")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


class env:
    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in KEYS}
        for k in KEYS:
            os.environ.pop(k, None)
        os.environ.update(self.kv)

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.fixture(scope="module")
def survey(port32):
    """The bench survey's model and two of its shots (the edge shot at column 0 and one in the
    middle), with the oracle's results for them."""
    vp = M.layered_model(NZ, NX, seed=0, water_rows=WATER)
    rho = M.gardner(vp, water_rows=WATER)
    vp0 = M.smooth_model(vp, 15.0, water_rows=WATER)
    rho0 = M.gardner(vp0, water_rows=WATER)
    src = M.ricker(NT, DT, 10.0, 0.15)
    sv = M.line_survey(NZ, NX, DX, DX, DT, NT, 60, src, spacing_cells=12, first_cell=0, sdepth_cells=1,
                       gdepth_cells=1)
    shots = M.survey_shots(sv)
    shots = [shots[0], shots[37]]
    assert all(len(s.igx) == NX for s in shots) and port32.checkpoint_interval(NT) == 89
    P = ITER
    obs, _ = port32.propagation(vp, rho, shots, DX, DX, DT, NT, PML, FS, 0.0, 2.0, 1, 0)
    adj, grad = port32.propagation(vp0, rho0, shots, DX, DX, DT, NT, PML, FS, P["freq"], 2.0, 1, 1, obs=obs)
    # the line search of acoustic2d_fwi.c:418-465, composed from the oracle's operations
    slow = np.where(vp0 != 0, 1.0 / vp0, 0).astype(np.float32)
    g = port32.smooth2d(port32.smooth2d(grad, P["rz"], 1), P["rx"], 0)
    fun1 = port32.objective(adj)
    scalar, pert = port32.model_perturbation(0.01, slow, g)
    lim = (P["waterdepth"], P["vp_water"], P["rho_water"], P["vpmin"], P["vpmax"], P["rhomin"], P["rhomax"])
    vpt, rhot = port32.fwi_trial(slow, pert, *lim)
    res, _ = port32.propagation(vpt, rhot, shots, DX, DX, DT, NT, PML, FS, P["freq"], 2.0, 1, 2, obs=obs)
    fun2 = port32.objective(res)
    steplen = port32.step_length(adj, res)
    _, vp2, rho2 = port32.fwi_update(slow, vp0, rho0, pert, steplen, *lim)
    return dict(vp=vp, rho=rho, vp0=vp0, rho0=rho0, shots=shots, obs=obs, adj=adj, grad=grad, vpt=vpt, rhot=rhot,
                res=res, fun1=fun1, fun2=fun2, steplen=steplen, scalar=scalar, vp2=vp2, rho2=rho2)


def _run(S, vp, rho, problem, path, obs=None):
    return E.propagation(vp, rho, S["shots"], DX, DX, DT, NT, PML, FS, 10.0, 2.0, 1, problem, obs=obs, path=path)


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_forward_seismograms(survey, path):
    S = survey
    got, _ = _run(S, S["vp"], S["rho"], 0, path)
    for i, (a, b) in enumerate(zip(got, S["obs"])):
        assert np.array_equal(a, b), f"shot {i}: rel-L2 {rel(a, b):.2e}"


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_gradient_and_adjoint_sources(survey, path):
    S = survey
    adj, grad = _run(S, S["vp0"], S["rho0"], 1, path, obs=S["obs"])
    for i, (a, b) in enumerate(zip(adj, S["adj"])):
        assert np.array_equal(a, b), f"shot {i}: rel-L2 {rel(a, b):.2e}"
    # FP64 stacks in tree order: within 1e-6 (bit-exact in practice)
    assert rel(grad, S["grad"]) <= 1e-6


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_line_search_residuals(survey, path):
    S = survey
    res, _ = _run(S, S["vpt"], S["rhot"], 2, path, obs=S["obs"])
    for i, (a, b) in enumerate(zip(res, S["res"])):
        assert np.array_equal(a, b), f"shot {i}: rel-L2 {rel(a, b):.2e}"


def test_fwi_iteration(survey):
    """fwi_ctx_fwi_iteration (gradient, smoothing, perturbation, trial model, line-search forward,
    misfits, step length, update) against the oracle composed step by step."""
    S = survey
    ctx = E.Context(0)
    try:
        ctx.set_model(S["vp0"], S["rho0"], DX, DX, DT, NT, PML, FS)
        ctx.set_shots(S["shots"])
        ctx.set_observed(S["obs"])
        r = ctx.fwi_iteration(E.IterParams(path=E.PATH_BATCHED, **ITER))
        vp_g, rho_g = ctx.model()
    finally:
        ctx.close()
    assert np.float32(r["fun1"]) == np.float32(S["fun1"])
    assert np.float32(r["fun2"]) == np.float32(S["fun2"])
    assert np.float32(r["scalar"]) == np.float32(S["scalar"])
    assert abs(r["steplen"] - S["steplen"]) <= 1e-6 * abs(S["steplen"])
    assert rel(vp_g, S["vp2"]) <= 1e-6 and rel(rho_g, S["rho2"]) <= 1e-6


def test_gradient_against_reference_build(survey):
    """The reference itself (strict-IEEE build of the unmodified sources) on the same two shots."""
    import pyoracle
    if not pyoracle.ref_available("strict"):
        pytest.skip("reference build not present")
    S = survey
    ref = pyoracle.Reference("strict")
    radj, rgrad = ref.propagation(S["vp0"], S["rho0"], S["shots"], DX, DX, DT, NT, PML, FS, 10.0, 2.0, 1, 1,
                                  obs=S["obs"])
    adj, grad = _run(S, S["vp0"], S["rho0"], 1, "batched", obs=S["obs"])
    for i, (a, b) in enumerate(zip(adj, radj)):
        assert np.array_equal(a, b), f"shot {i}: rel-L2 {rel(a, b):.2e}"
    assert rel(grad, rgrad) <= 1e-6


def _ctx_run(S, vp, rho, problem, path, obs=None):
    """The native context API (a fresh context reads FWI_MATH when it is created)."""
    ctx = E.Context(0)
    try:
        ctx.set_model(vp, rho, DX, DX, DT, NT, PML, FS)
        ctx.set_shots(S["shots"])
        if obs is not None:
            ctx.set_observed(obs)
        ctx.run(problem, 10.0, 2, 1, E.PATH_PLAIN if path == "plain" else E.PATH_BATCHED)
        return [ctx.traces(i) for i in range(len(S["shots"]))], (ctx.gradient() if problem == 1 else None)
    finally:
        ctx.close()


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_contracted_math(survey, path):
    """FWI_MATH=1 (packed FMAs) at full size: seismograms within rel-L2 1e-5, adjoint sources,
    line-search residuals and gradient within 1e-4 of the bit-exact FP32 results."""
    S = survey
    with env(FWI_MATH="1"):
        pre, _ = _ctx_run(S, S["vp"], S["rho"], 0, path)
        adj, grad = _ctx_run(S, S["vp0"], S["rho0"], 1, path, obs=S["obs"])
        res, _ = _ctx_run(S, S["vpt"], S["rhot"], 2, path, obs=S["obs"])
    for i in range(len(S["shots"])):
        assert rel(pre[i], S["obs"][i]) <= 1e-5
        assert rel(adj[i], S["adj"][i]) <= 1e-4
        assert rel(res[i], S["res"][i]) <= 1e-4
    assert rel(grad, S["grad"]) <= 1e-4
