"""The CUDA engine against the oracle beyond the golden cases: the per-shot engine
entry point with its checkpoint object, the FWI-loop operations, the batched path
against the plain one at the survey's full size, a full-size forward shot against
the oracle, errors and the device-memory budget."""
import ctypes as C
import os

import numpy as np
import pytest

from fwiedu import engine as E
from fwiedu import models as M
from golden_cases import Case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _rec(shot, traces, keep):
    return E.make_records([shot], [traces], keep)


def test_engine_entry_point_modes(port32):
    """iso_acoustic2d_propagation_engine with the checkpoint life cycle of propagation.c:903-978."""
    c = Case("fs1_small")
    L = E.lib()
    s = c.shots[1]  # the shot with a narrow window
    vpw = np.ascontiguousarray(c.vp0[s.ix_min:s.ix_max + 1])
    rhow = np.ascontiguousarray(c.rho0[s.ix_min:s.ix_max + 1])
    nxx = vpw.shape[0]
    keep = []
    tr = np.zeros((len(s.igx), s.ns), np.float32)
    rec = _rec(s, tr, keep)
    chk = (C.c_byte * 64)()
    L.acoustic2dCheckPoint_init(chk)
    L.alloc_acoustic2dCheckPoint(chk, c.nz + 2 * c.pml, nxx + 2 * c.pml, c.nt)
    prec = np.zeros((nxx, c.nz), np.float32)
    rc = L.fwi_iso_acoustic2d_propagation_engine(rec, chk, E.rows(vpw), E.rows(rhow), nxx, c.nz, C.c_float(c.dx),
                                                 C.c_float(c.dx), C.c_float(c.dt), c.nt, c.pml, c.fs, 1, 1, 1, 0,
                                                 E.rows(prec))
    assert rc == 0, L.fwi_last_error()
    # mode 1 samples the same traces as a forward run of this shot's window
    want = port32.forward(s, c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    assert np.array_equal(tr, want)
    assert np.isfinite(prec).all() and prec.max() > 0
    # mode 2 from an adjoint source written into the same record
    tr[:] = c.adj[1]
    g = np.zeros((nxx, c.nz), np.float32)
    rc = L.fwi_iso_acoustic2d_propagation_engine(rec, chk, E.rows(vpw), E.rows(rhow), nxx, c.nz, C.c_float(c.dx),
                                                 C.c_float(c.dx), C.c_float(c.dt), c.nt, c.pml, c.fs, 1, 2, 1, 0,
                                                 E.rows(g))
    assert rc == 0, L.fwi_last_error()
    # the oracle's per-shot gradient without preconditioning is the same raw mode-2 gradient
    gs = np.zeros((nxx, c.nz), np.float32)
    pre = c.obs[1].copy()
    import pyoracle
    lib = port32.lib
    shot = port32._shot(s)
    rc = lib.orc_shot_gradient(C.byref(shot), c.vp0.ctypes.data_as(C.POINTER(C.c_float)),
                               c.rho0.ctypes.data_as(C.POINTER(C.c_float)), c.nz, c.nx, C.c_float(c.dx),
                               C.c_float(c.dx), C.c_float(c.dt), c.nt, c.pml, c.fs, C.c_float(10.0), 2, 0,
                               np.ascontiguousarray(c.obs[1]).ctypes.data_as(C.POINTER(C.c_float)),
                               pre.ctypes.data_as(C.POINTER(C.c_float)), gs.ctypes.data_as(C.POINTER(C.c_float)), None)
    assert rc == 0
    assert np.array_equal(g, gs)
    L.free_acoustic2dCheckPoint(chk)


def test_fwi_loop_operations_match_reference():
    c = Case("fs1_small")
    L = E.lib()
    L.calculate_objective_value.restype = C.c_float
    L.calculate_step_length.restype = C.c_float
    L.compute_model_perturbation.restype = C.c_float
    keep = []
    ra = E.make_records(c.shots, [a.copy() for a in c.adj], keep)
    rr = E.make_records(c.shots, [a.copy() for a in c.res], keep)
    assert np.float32(L.calculate_objective_value(ra, c.nshot)) == c["fun1"]
    assert np.float32(L.calculate_step_length(ra, rr, c.nshot)) == c["steplen"]
    g = np.ascontiguousarray(c.grad)
    t = np.zeros_like(g)
    out = np.zeros_like(g)
    L.smooth2D(E.rows(g), E.rows(t), c.nx, c.nz, 1, 1)
    L.smooth2D(E.rows(t), E.rows(out), c.nx, c.nz, 1, 0)
    assert np.array_equal(out, c["grad_smooth"])
    slow = (1.0 / c.vp0).astype(np.float32)
    pert = np.zeros_like(g)
    fp = C.POINTER(C.c_float)
    sc = L.compute_model_perturbation(C.c_float(0.01), slow.ctypes.data_as(fp), out.ctypes.data_as(fp),
                                      pert.ctypes.data_as(fp), g.size)
    assert np.float32(sc) == c["pert_scalar"]
    assert np.array_equal(pert, c["perturb"])


def test_adjoint_source_entry_point():
    c = Case("fs1_small")
    L = E.lib()
    keep = []
    pre = [np.zeros_like(o) for o in c.obs]
    # predicted data of the smoothed model are the residual plus the observed data only before the taper;
    # recompute them with the engine, then form the adjoint source through the drop-in
    p, _ = E.propagation(c.vp0, c.rho0, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 0.0, 2.0, 1, 0)
    for i in range(c.nshot):
        rp = E.make_records([c.shots[i]], [p[i].copy()], keep)
        ro = E.make_records([c.shots[i]], [c.obs[i].copy()], keep)
        out = np.zeros_like(p[i])
        ra = E.make_records([c.shots[i]], [out], keep)
        L.compute_adjoint_source2d(rp, ro, E.rows(c.vp0), C.c_float(10.0), 2, ra)
        assert np.array_equal(out, c.adj[i]), f"shot {i}"


def test_batched_equals_plain_full_size():
    """The survey geometry at full size (221 x 601, 40-cell layer, free surface): 2 shots, short record."""
    nz, nx, nt = 221, 601, 600
    vp = M.layered_model(nz, nx, seed=0)
    rho = M.gardner(vp)
    src = M.ricker(nt, 0.001, 10.0, 0.15)
    sv = M.line_survey(nz, nx, 12.5, 12.5, 0.001, nt, 2, src, spacing_cells=300, first_cell=100)
    shots = M.survey_shots(sv)
    a, _ = E.propagation(vp, rho, shots, 12.5, 12.5, 0.001, nt, 40, 1, 0.0, 2.0, 1, 0, path="plain")
    b, _ = E.propagation(vp, rho, shots, 12.5, 12.5, 0.001, nt, 40, 1, 0.0, 2.0, 1, 0, path="batched")
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    vp0 = M.smooth_model(vp, 15.0)
    rho0 = M.gardner(vp0)
    ga = E.propagation(vp0, rho0, shots, 12.5, 12.5, 0.001, nt, 40, 1, 10.0, 2.0, 1, 1, obs=a, path="plain")
    gb = E.propagation(vp0, rho0, shots, 12.5, 12.5, 0.001, nt, 40, 1, 10.0, 2.0, 1, 1, obs=a, path="batched")
    assert all(np.array_equal(x, y) for x, y in zip(ga[0], gb[0]))
    assert np.array_equal(ga[1], gb[1])


def test_full_size_forward_shot_matches_oracle(port32):
    """One shot of the 221 x 601 survey model, nt = 4001, against the oracle: bit for bit."""
    nz, nx, nt = 221, 601, 4001
    vp = M.layered_model(nz, nx, seed=0)
    rho = M.gardner(vp)
    src = M.ricker(nt, 0.001, 10.0, 0.15)
    sv = M.line_survey(nz, nx, 12.5, 12.5, 0.001, nt, 1, src, spacing_cells=1, first_cell=300)
    shots = M.survey_shots(sv)
    g, _ = E.propagation(vp, rho, shots, 12.5, 12.5, 0.001, nt, 40, 1, 0.0, 2.0, 1, 0, path="batched")
    o = port32.forward(shots[0], vp, rho, 12.5, 12.5, 0.001, nt, 40, 1)
    assert np.array_equal(g[0], o)


def test_errors_and_budget():
    c = Case("fs1_small")
    ctx = E.Context(0)
    with pytest.raises(E.FwiError) as e:
        ctx.set_model(c.vp, c.rho, c.dx, c.dx, c.dt, c.nt, 2, 1)  # free surface needs pml >= 3
    assert e.value.code == E.FWI_ERR_ARG
    ctx.set_model(c.vp, c.rho, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    bad = Case("fs1_small").shots[:1]
    bad[0].isz = c.nz + 5
    with pytest.raises(E.FwiError):
        ctx.set_shots(bad)
    with pytest.raises(E.FwiError) as e:
        ctx.run(3)
    assert e.value.code == E.FWI_ERR_ARG
    ctx.close()
    small = E.Context(0, budget_bytes=1 << 20)
    small.set_model(c.vp, c.rho, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    small.set_shots(Case("fs1_small").shots)
    with pytest.raises(E.FwiError) as e:
        small.run(1, 10.0, 2, 1)
    assert e.value.code == E.FWI_ERR_NOMEM
    small.close()


def test_context_api_gradient_and_objective(port32):
    c = Case("noprec")
    ctx = E.Context(0)
    ctx.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    ctx.set_shots(c.shots)
    ctx.set_observed(c.obs)
    ctx.run(1, 10.0, 2, c.precondition, E.PATH_BATCHED)
    assert rel(ctx.gradient(), c.grad) <= 1e-6
    for i in range(c.nshot):
        assert np.array_equal(ctx.traces(i), c.adj[i])
    assert np.float32(ctx.objective()) == c["fun1"]
    st = ctx.stats()
    assert st["kernel_launches"] > c.nt and st["cell_updates"] > 0
    ctx.close()


def test_fwi_iteration_matches_oracle(port32):
    """fwi_ctx_fwi_iteration against the oracle composed step by step (acoustic2d_fwi.c:411-465)."""
    c = Case("fs1_small")
    P = dict(rx=2, rz=1, precondition=1, filter=2, freq=10.0, waterdepth=6, vp_water=1500.0, rho_water=1000.0,
             vpmin=1500.0, vpmax=4700.0, rhomin=1000.0, rhomax=2700.0, gardner=1)
    ctx = E.Context(0)
    ctx.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
    ctx.set_shots(c.shots)
    ctx.set_observed(c.obs)
    r = ctx.fwi_iteration(E.IterParams(path=E.PATH_BATCHED, **P))
    vp_g, rho_g = ctx.model()
    ctx.close()
    # oracle
    slow = np.where(c.vp0 != 0, 1.0 / c.vp0, 0).astype(np.float32)
    pre0, grad = port32.propagation(c.vp0, c.rho0, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 10.0, 2.0, 1, 1,
                                    obs=c.obs)
    g = port32.smooth2d(port32.smooth2d(grad, P["rz"], 1), P["rx"], 0)
    fun1 = port32.objective(pre0)
    scalar, pert = port32.model_perturbation(0.01, slow, g)
    vpt, rhot = port32.fwi_trial(slow, pert, 6, 1500.0, 1000.0, 1500.0, 4700.0, 1000.0, 2700.0)
    pre1, _ = port32.propagation(vpt, rhot, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 10.0, 2.0, 1, 2, obs=c.obs)
    fun2 = port32.objective(pre1)
    steplen = port32.step_length(pre0, pre1)
    slow2, vp2, rho2 = port32.fwi_update(slow, c.vp0, c.rho0, pert, steplen, 6, 1500.0, 1000.0, 1500.0, 4700.0,
                                         1000.0, 2700.0)
    assert np.float32(r["fun1"]) == np.float32(fun1)
    assert np.float32(r["fun2"]) == np.float32(fun2)
    assert np.float32(r["scalar"]) == np.float32(scalar)
    assert abs(r["steplen"] - steplen) <= 1e-6 * abs(steplen)
    assert rel(vp_g, vp2) <= 1e-6 and rel(rho_g, rho2) <= 1e-6


def test_bounded_wait_gives_up_and_context_survives():
    """The step kernel's mbarrier waits are bounded: a wait on a phase that nothing completes gives
    up after its limit, the kernel sets the error word and returns, the host reports FWI_ERR_CUDA,
    and the same context then runs a golden case bit for bit (no fault, no hang, no reset)."""
    c = Case("fs1_small")
    ctx = E.Context(0)
    try:
        L = E.lib()
        assert L.fwi_ctx_selftest_wait(ctx.h, 50) == E.FWI_ERR_CUDA
        assert b"did not complete" in L.fwi_last_error()
        assert L.fwi_ctx_selftest_wait(ctx.h, 0) == E.FWI_ERR_ARG
        ctx.set_model(c.vp, c.rho, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
        ctx.set_shots(c.shots)
        ctx.run(0, path=E.PATH_BATCHED)
        for i in range(c.nshot):
            assert np.array_equal(ctx.traces(i), c.obs[i])
    finally:
        ctx.close()
