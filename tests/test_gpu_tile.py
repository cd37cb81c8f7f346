"""The TMA-fed step kernels in all of their launch shapes.

Forward passes of two or more shots can run as one persistent wavefront launch (fwi_wave.cuh,
FWI_PERSIST=1; off by default and in the shape tests).  The step launches' shape is tuned per
grid and shot count: the halo depth (one step per launch, or two with the temporal-blocking
kernel), the tile width (8 or 16 columns, one-step kernel), the depth of the shared-memory stage
ring (2 to 4 shots in flight) and the number of shots each block walks; environment variables
override the choice (FWI_DEPTH pins the halo depth).  Every shape must give the same bits: the
reference's golden seismograms and gradient, and -- on a 12-shot survey where blocks walk more
shots than the ring has stages -- the results of the previous cp.async kernel.  The
contracted-FMA mode is held to the stated FP32 tolerance instead.
"""
import os

import numpy as np
import pytest

from fwiedu import engine as E
from fwiedu import models as M
from golden_cases import Case

pytestmark = pytest.mark.gpu

SHAPES = [
    # the one-step kernel (the default) and the two-step kernel (temporal blocking)
    {},
    {"FWI_DEPTH": "2"},
    {"FWI_DEPTH": "2", "FWI_NST": "3"},
    {"FWI_DEPTH": "2", "FWI_NST": "2", "FWI_CHUNK": "1"},
    {"FWI_DEPTH": "2", "FWI_NST": "3", "FWI_CHUNK": "5"},
    {"FWI_DEPTH": "2", "FWI_NST": "2", "FWI_CHUNK": "32"},
    # the one-step kernel in its launch shapes
    {"FWI_DEPTH": "1"},
    {"FWI_DEPTH": "1", "FWI_TX": "8"},
    {"FWI_DEPTH": "1", "FWI_TX": "16", "FWI_NST": "2", "FWI_CHUNK": "1"},
    {"FWI_DEPTH": "1", "FWI_TX": "8", "FWI_NST": "2", "FWI_CHUNK": "3"},
    {"FWI_DEPTH": "1", "FWI_TX": "16", "FWI_NST": "4", "FWI_CHUNK": "2"},
    {"FWI_DEPTH": "1", "FWI_TX": "16", "FWI_NST": "3", "FWI_CHUNK": "32"},
    {"FWI_DEPTH": "1", "FWI_GPT": "2"},
    {"FWI_DEPTH": "1", "FWI_TX": "8", "FWI_GPT": "2", "FWI_NST": "3", "FWI_CHUNK": "5"},
    {"FWI_DEPTH": "1", "FWI_TX": "16", "FWI_GPT": "2", "FWI_NST": "2", "FWI_CHUNK": "1"},
    {"FWI_DEPTH": "1", "FWI_OCC": "3"},
    {"FWI_DEPTH": "1", "FWI_OCC": "3", "FWI_NST": "3", "FWI_CHUNK": "8"},
    {"FWI_DEPTH": "1", "FWI_OCC": "3", "FWI_NST": "2", "FWI_CHUNK": "1"},
]
KEYS = ("FWI_TX", "FWI_NST", "FWI_CHUNK", "FWI_KERNEL", "FWI_MATH", "FWI_TUNE", "FWI_GPT", "FWI_OCC", "FWI_DEPTH",
        "FWI_PERSIST")


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
        # the shapes are those of the step launches: forward passes too unless a case asks for
        # the persistent wavefront launch
        os.environ["FWI_PERSIST"] = "0"
        os.environ.update(self.kv)

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def run_case(vp, rho, dx, dt, nt, pml, fs, shots, obs=None, precondition=1, path=E.PATH_BATCHED):
    ctx = E.Context(0)
    try:
        ctx.set_model(vp, rho, dx, dx, dt, nt, pml, fs)
        ctx.set_shots(shots)
        if obs is None:
            ctx.run(0, path=path)
            return [ctx.traces(i) for i in range(len(shots))], None
        ctx.set_observed(obs)
        ctx.run(1, 10.0, 2, precondition, path)
        return [ctx.traces(i) for i in range(len(shots))], ctx.gradient()
    finally:
        ctx.close()


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: ",".join(f"{k[4:]}={v}" for k, v in s.items()) or "auto")
def test_shapes_match_golden(shape):
    c = Case("fs1_small")
    with env(**shape):
        pre, _ = run_case(c.vp, c.rho, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots)
        adj, grad = run_case(c.vp0, c.rho0, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots, obs=c.obs)
    for i in range(c.nshot):
        assert np.array_equal(pre[i], c.obs[i]), f"shot {i}"
        assert np.array_equal(adj[i], c.adj[i]), f"adjoint source {i}"
    assert rel(grad, c.grad) <= 1e-6
    assert np.mean(grad == c.grad) > 0.999


def survey12(nt=320):
    nz, nx = 90, 240
    vp = M.layered_model(nz, nx, seed=3)
    rho = M.gardner(vp)
    src = M.ricker(nt, 0.001, 12.0, 0.1)
    sv = M.line_survey(nz, nx, 10.0, 10.0, 0.001, nt, 12, src, spacing_cells=19, first_cell=5)
    return vp, rho, M.survey_shots(sv), nt


def test_pipeline_wraps_bit_identical_to_cp_async_kernel():
    vp, rho, shots, nt = survey12()
    with env(FWI_KERNEL="step"):
        obs, _ = run_case(vp, rho, 10.0, 0.001, nt, 20, 1, shots)
    vp0 = M.smooth_model(vp, 8.0)
    rho0 = M.gardner(vp0)
    with env(FWI_KERNEL="step"):
        adj_ref, grad_ref = run_case(vp0, rho0, 10.0, 0.001, nt, 20, 1, shots, obs=obs)
    for shape in SHAPES[1:]:
        with env(**shape):
            pre, _ = run_case(vp, rho, 10.0, 0.001, nt, 20, 1, shots)
            adj, grad = run_case(vp0, rho0, 10.0, 0.001, nt, 20, 1, shots, obs=obs)
        assert all(np.array_equal(a, b) for a, b in zip(pre, obs)), shape
        assert all(np.array_equal(a, b) for a, b in zip(adj, adj_ref)), shape
        assert np.array_equal(grad, grad_ref), shape


def test_plain_path_single_shot_tiles():
    vp, rho, shots, nt = survey12(200)
    with env(FWI_KERNEL="step"):
        want, _ = run_case(vp, rho, 10.0, 0.001, nt, 20, 0, shots[:3], path=E.PATH_PLAIN)
    got, _ = run_case(vp, rho, 10.0, 0.001, nt, 20, 0, shots[:3], path=E.PATH_PLAIN)
    assert all(np.array_equal(a, b) for a, b in zip(got, want))


def test_contracted_math_within_tolerance():
    """FWI_MATH=1 against the reference's golden vectors: seismograms within rel-L2 1e-5,
    gradient within 1e-4.  (This case is well conditioned: its FP32 and FP64 gradients
    agree to 5e-6.  The 12-shot survey above is not -- its residual is 1e-4 of the data --
    so it only serves the bitwise comparisons.)"""
    c = Case("fs1_small")
    with env(FWI_MATH="1"):
        pre, _ = run_case(c.vp, c.rho, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots)
        adj, grad = run_case(c.vp0, c.rho0, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots, obs=c.obs)
    for i in range(c.nshot):
        assert rel(pre[i], c.obs[i]) <= 1e-5
        assert rel(adj[i], c.adj[i]) <= 1e-4
    assert rel(grad, c.grad) <= 1e-4


def test_autotuned_shape_is_bit_identical_and_cached():
    """The autotuner times launch shapes on the run's own scratch frames: the run it precedes
    must give the same bits as with the heuristic shape, and the shape is kept for the process."""
    c = Case("fs1_small")
    with env(FWI_TUNE="0"):
        ref_pre, _ = run_case(c.vp, c.rho, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots)
        ref_adj, ref_grad = run_case(c.vp0, c.rho0, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots, obs=c.obs)
    with env():
        pre, _ = run_case(c.vp, c.rho, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots)
        adj, grad = run_case(c.vp0, c.rho0, c.dx, c.dt, c.nt, c.pml, c.fs, c.shots, obs=c.obs)
        ctx = E.Context(0)
        ctx.set_model(c.vp, c.rho, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
        ctx.set_shots(c.shots)
        ctx.run(0, path=E.PATH_BATCHED)
        L = E.lib()
        import ctypes as C
        tx, nst, ch = C.c_int(), C.c_int(), C.c_int()
        L.fwi_ctx_launch_shape(ctx.h, C.byref(tx), C.byref(nst), C.byref(ch))
        ctx.close()
    assert tx.value in (8, 16) and 2 <= nst.value <= 4 and 1 <= ch.value <= c.nshot
    assert all(np.array_equal(a, b) for a, b in zip(pre, ref_pre))
    assert all(np.array_equal(a, b) for a, b in zip(adj, ref_adj))
    assert np.array_equal(grad, ref_grad)


def test_many_receivers_match_cp_async_kernel():
    """More receivers than one pass of the sampling blocks covers (a shallow model has one tile
    of rows, so 288 gathers per pass against 1500 receivers): every trace sample is the cp.async
    kernel's, bit for bit, in both compiled variants and the narrow tiles."""
    nz, nx, nt = 30, 1500, 120
    vp = M.layered_model(nz, nx, seed=11, water_rows=4)
    rho = M.gardner(vp, water_rows=4)
    src = M.ricker(nt, 0.001, 15.0, 0.06)
    sv = M.line_survey(nz, nx, 10.0, 10.0, 0.001, nt, 3, src, spacing_cells=400, first_cell=100)
    shots = M.survey_shots(sv)
    assert all(len(s.igx) == nx for s in shots)  # a receiver in every column
    with env(FWI_KERNEL="step"):
        ref, _ = run_case(vp, rho, 10.0, 0.001, nt, 10, 1, shots)
    for shape in ({}, {"FWI_DEPTH": "2"}, {"FWI_DEPTH": "1", "FWI_OCC": "3"}, {"FWI_DEPTH": "1", "FWI_TX": "8"}):
        with env(**shape):
            got, _ = run_case(vp, rho, 10.0, 0.001, nt, 10, 1, shots)
        for i, (a, b) in enumerate(zip(got, ref)):
            assert np.array_equal(a, b), (shape, i)


def run_persistent(vp, rho, dx, dt, nt, pml, fs, shots, obs=None):
    """run_case with the wavefront launch on (it runs one step per launch, so the callers pin the
    halo depth the tuner would otherwise choose); also returns whether the pass used it"""
    ctx = E.Context(0)
    try:
        ctx.set_model(vp, rho, dx, dx, dt, nt, pml, fs)
        ctx.set_shots(shots)
        if obs is None:
            ctx.run(0, path=E.PATH_BATCHED)
            return [ctx.traces(i) for i in range(len(shots))], None, ctx.launch_shape()["persistent"]
        ctx.set_observed(obs)
        ctx.run(1, 10.0, 2, 1, E.PATH_BATCHED)
        return [ctx.traces(i) for i in range(len(shots))], ctx.gradient(), None
    finally:
        ctx.close()


def test_wavefront_matches_golden():
    """The persistent forward launch against the reference's golden seismograms and adjoint sources
    (the two shots of the case whose windows span the model form one group; the third shot's
    window differs), and its gradient -- whose checkpointing forward with the pseudo-Hessian runs
    as the wavefront launch -- against the step launches', bit for bit."""
    c = Case("fs1_small")
    pick = [0, 2]
    shots = [c.shots[i] for i in pick]
    obs = [c.obs[i] for i in pick]
    with env(FWI_PERSIST="1", FWI_DEPTH="1"):
        pre, _, used = run_persistent(c.vp, c.rho, c.dx, c.dt, c.nt, c.pml, c.fs, shots)
        adj, grad, _ = run_persistent(c.vp0, c.rho0, c.dx, c.dt, c.nt, c.pml, c.fs, shots, obs=obs)
    with env(FWI_PERSIST="0"):
        _, grad_ref = run_case(c.vp0, c.rho0, c.dx, c.dt, c.nt, c.pml, c.fs, shots, obs=obs)
    assert used == 1
    for k, i in enumerate(pick):
        assert np.array_equal(pre[k], c.obs[i]), f"shot {i}"
        assert np.array_equal(adj[k], c.adj[i]), f"adjoint source {i}"
    assert np.array_equal(grad, grad_ref)


@pytest.mark.parametrize("nshot", [2, 5, 12])
def test_wavefront_matches_step_launches(nshot):
    """Shot ranges of 2..n shots, several z-tiles and the receiver and source tiles: seismograms,
    adjoint sources and gradient of the wavefront launch equal the step launches' bit for bit."""
    vp, rho, shots, nt = survey12()
    shots = shots[:nshot]
    vp0 = M.smooth_model(vp, 8.0)
    rho0 = M.gardner(vp0)
    with env(FWI_PERSIST="0"):
        obs, _ = run_case(vp, rho, 10.0, 0.001, nt, 20, 1, shots)
        adj_ref, grad_ref = run_case(vp0, rho0, 10.0, 0.001, nt, 20, 1, shots, obs=obs)
    with env(FWI_PERSIST="1", FWI_DEPTH="1"):
        pre, _, used = run_persistent(vp, rho, 10.0, 0.001, nt, 20, 1, shots)
        adj, grad, _ = run_persistent(vp0, rho0, 10.0, 0.001, nt, 20, 1, shots, obs=obs)
    assert used == 1
    assert all(np.array_equal(a, b) for a, b in zip(pre, obs))
    assert all(np.array_equal(a, b) for a, b in zip(adj, adj_ref))
    assert np.array_equal(grad, grad_ref)


def test_wavefront_many_receivers():
    """1500 receivers, one per column, on a shallow model: every sample taken inside the tiles
    equals the step launches' sampling column, bit for bit."""
    nz, nx, nt = 30, 1500, 120
    vp = M.layered_model(nz, nx, seed=11, water_rows=4)
    rho = M.gardner(vp, water_rows=4)
    src = M.ricker(nt, 0.001, 15.0, 0.06)
    sv = M.line_survey(nz, nx, 10.0, 10.0, 0.001, nt, 3, src, spacing_cells=400, first_cell=100)
    shots = M.survey_shots(sv)
    with env(FWI_PERSIST="0"):
        ref, _ = run_case(vp, rho, 10.0, 0.001, nt, 10, 1, shots)
    with env(FWI_PERSIST="1", FWI_DEPTH="1"):
        got, _, used = run_persistent(vp, rho, 10.0, 0.001, nt, 10, 1, shots)
    assert used == 1
    for i, (a, b) in enumerate(zip(got, ref)):
        assert np.array_equal(a, b), i


def test_injection_with_several_receivers_per_column(port32):
    """Receivers in two rows of every even column and in one row of every odd column: an adjoint
    step injects the odd columns' receivers from the per-block receiver table and walks the list
    of the even columns (several receivers in one tile column), in the list's order.  Seismograms,
    adjoint sources and the gradient equal the oracle's bit for bit on the batched and the
    one-shot path (propagation.c:676-682)."""
    nz, nx, nt, dx, dt, pml, fs = 40, 70, 300, 10.0, 0.001, 10, 1
    vp = M.layered_model(nz, nx, seed=5, water_rows=4)
    rho = M.gardner(vp, water_rows=4)
    vp0 = M.smooth_model(vp, 4.0, water_rows=4)
    rho0 = M.gardner(vp0, water_rows=4)
    src = M.ricker(nt, dt, 15.0, 0.06)
    sv = M.line_survey(nz, nx, dx, dx, dt, nt, 2, src, spacing_cells=40, first_cell=15)
    gx = np.array([x for x in range(nx) for _ in range(2 if x % 2 == 0 else 1)], np.int32)
    gz = np.array([z for x in range(nx) for z in ((2, 6) if x % 2 == 0 else (3,))], np.int32)
    for k in range(len(sv.sx)):
        sv.gx[k] = gx.copy()
        sv.gz[k] = gz.copy()
    shots = M.survey_shots(sv)
    assert all(s.ntr == 105 for s in shots)
    obs, _ = port32.propagation(vp, rho, shots, dx, dx, dt, nt, pml, fs, 0.0, 2.0, 1, 0)
    adj, grad = port32.propagation(vp0, rho0, shots, dx, dx, dt, nt, pml, fs, 10.0, 2.0, 1, 1, obs=obs)
    for path in (E.PATH_BATCHED, E.PATH_PLAIN):
        pre, _ = run_case(vp, rho, dx, dt, nt, pml, fs, shots, path=path)
        got_adj, got_grad = run_case(vp0, rho0, dx, dt, nt, pml, fs, shots, obs=obs, path=path)
        for i in range(len(shots)):
            assert np.array_equal(pre[i], obs[i]), (path, "seismogram", i)
            assert np.array_equal(got_adj[i], adj[i]), (path, "adjoint source", i)
        assert np.array_equal(got_grad, grad), (path, "gradient")
