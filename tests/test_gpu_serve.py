"""The serving loop (fwi_server_*): requests of mixed grid sizes admitted by device-memory
footprint and batched continuously (the runs in flight share every step launch).  Every result
must be the same alone and in the mix -- here bit for bit, since each run keeps its own
deterministic state and the executor's arithmetic is the single run's -- and the reference's
golden vectors still hold for the requests that have them.  Admission must keep the admitted
footprint within the budget, and a request larger than the budget is refused at submission.
"""
import numpy as np
import pytest

from fwiedu import engine as E
from fwiedu import models as M
from golden_cases import Case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def mixed_requests():
    """Modeling and gradient requests on three grids, with the golden cases among them."""
    reqs = []
    for name in ("fs1_small", "noprec"):
        c = Case(name)
        reqs.append((name + "/model", E.REQ_MODEL, dict(vp=c.vp, rho=c.rho, dx=c.dx, dz=c.dx, dt=c.dt, nt=c.nt,
                                                        pml=c.pml, fs=c.fs, shots=c.shots, precondition=c.precondition)))
        reqs.append((name + "/grad", E.REQ_GRADIENT, dict(vp=c.vp0, rho=c.rho0, dx=c.dx, dz=c.dx, dt=c.dt, nt=c.nt,
                                                          pml=c.pml, fs=c.fs, shots=c.shots, obs=c.obs,
                                                          precondition=c.precondition)))
    nz, nx, nt = 60, 150, 400
    vp = M.layered_model(nz, nx, seed=21, water_rows=5, anom_sigma=4)
    rho = M.gardner(vp, water_rows=5)
    sv = M.line_survey(nz, nx, 10.0, 10.0, 0.001, nt, 4, M.ricker(nt, 0.001, 12.0, 0.08), spacing_cells=30,
                       first_cell=10)
    shots = M.survey_shots(sv)
    obs = [np.random.default_rng(i).standard_normal((len(s.igx), s.ns)).astype(np.float32) for i, s in enumerate(shots)]
    reqs.append(("big/model", E.REQ_MODEL, dict(vp=vp, rho=rho, dx=10.0, dz=10.0, dt=0.001, nt=nt, pml=12, fs=1,
                                                 shots=shots)))
    reqs.append(("big/grad", E.REQ_GRADIENT, dict(vp=vp, rho=rho, dx=10.0, dz=10.0, dt=0.001, nt=nt, pml=12, fs=1,
                                                  shots=shots, obs=obs)))
    return reqs


def run(server, reqs, together):
    out = {}
    if together:
        ids = {}
        for name, kind, kw in reqs:
            r, holder = E.request(kind, **kw)
            ids[name] = (server.submit(r, holder), r)
        for name, (rid, _) in ids.items():
            out[name] = server.wait(rid)
    else:
        for name, kind, kw in reqs:
            r, holder = E.request(kind, **kw)
            out[name] = server.wait(server.submit(r, holder))
    return out


def test_results_same_alone_and_in_the_mix():
    reqs = mixed_requests()
    alone = E.Server(0, 0, max_active=1)
    a = run(alone, reqs, together=False)
    alone.close()
    mix = E.Server(0, 0, max_active=4)
    b = run(mix, reqs * 2, together=True)  # each request twice, all in flight together
    rep = mix.report()
    mix.close()
    assert rep["completed"] == 2 * len(reqs) and rep["failed"] == 0
    assert rep["peak_active"] >= 2  # they did overlap
    for name, _, _ in reqs:
        assert a[name]["status"] == 0 and b[name]["status"] == 0, (a[name]["error"], b[name]["error"])
        for x, y in zip(a[name]["traces"], b[name]["traces"]):
            assert np.array_equal(x, y), name
        if a[name]["grad"] is not None:
            assert np.array_equal(a[name]["grad"], b[name]["grad"]), name
            assert a[name]["objective"] == b[name]["objective"]
    # the golden cases inside the mix are still the reference's results
    c = Case("fs1_small")
    assert all(np.array_equal(x, y) for x, y in zip(b["fs1_small/model"]["traces"], c.obs))
    assert all(np.array_equal(x, y) for x, y in zip(b["fs1_small/grad"]["traces"], c.adj))
    assert rel(b["fs1_small/grad"]["grad"], c.grad) <= 1e-6
    assert rep["p99_ms"] >= rep["p50_ms"] > 0


def test_admission_keeps_within_budget():
    reqs = mixed_requests()
    sizes = []
    probe = E.Server(0, 0, max_active=1)
    for name, kind, kw in reqs:
        r, _ = E.request(kind, **kw)
        sizes.append(probe.bytes(r))
    probe.close()
    budget = int(max(sizes) * 1.5)  # room for the largest request and part of another
    srv = E.Server(0, budget, max_active=4)
    run(srv, reqs * 2, together=True)
    rep = srv.report()
    srv.close()
    assert rep["completed"] == 2 * len(reqs)
    assert rep["peak_bytes"] <= budget
    assert rep["budget"] == budget


def test_oversize_request_is_refused():
    c = Case("fs1_small")
    srv = E.Server(0, 1 << 20, max_active=2)  # 1 MiB: nothing fits
    r, holder = E.request(E.REQ_GRADIENT, vp=c.vp0, rho=c.rho0, dx=c.dx, dz=c.dx, dt=c.dt, nt=c.nt, pml=c.pml,
                          fs=c.fs, shots=c.shots, obs=c.obs)
    with pytest.raises(E.FwiError) as e:
        srv.submit(r, holder)
    assert e.value.code == E.FWI_ERR_NOMEM
    assert srv.report()["rejected"] == 1
    srv.close()


def test_estimate_covers_what_a_run_allocates():
    for name in ("fs1_small", "filt0"):
        c = Case(name)
        ctx = E.Context(0)
        ctx.set_model(c.vp0, c.rho0, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs)
        ctx.set_shots(c.shots)
        ctx.set_observed(c.obs)
        ctx.run(1, 10.0, int(c.filter), c.precondition, E.PATH_BATCHED)
        used = ctx.stats()["device_bytes"]
        ctx.close()
        est = E.estimate_bytes(c.shots, c.nz, c.nx, c.nt, c.pml, 1, int(c.filter))
        assert used <= est, (name, used, est)
