"""Physics known-answer tests of the algorithm the engine reproduces, on the oracle's FP64 build.

The reference ships no expected outputs, so besides its own runs (the golden vectors) the
algorithm is held to two properties of the wave equation it discretises:

* reciprocity: with the source and the receiver in the same homogeneous layer (the same K and
  rho at both points, so that the source scaling K*dt^2/(dx*dz) of propagation.c:558 is the
  same), exchanging them leaves the pressure trace unchanged up to the discretisation error of
  the variable-density operator (propagation.c:13-74), with and without the free surface;
* the gradient (propagation.c:633-744, imaging every fifth step, scaled by 2/(rho v): the
  derivative of the misfit with respect to slowness at fixed density) agrees with central
  finite differences of the misfit (optimization.c:99-132) along smooth perturbations below the
  water layer: same sign in every direction, the misfit linear in the step, and one scale
  factor for all directions within the discretisation error of the adjoint-state gradient
  (measured 2.1e-3 to 2.5e-3 at 6 Hz, within 13 % of their mean; at 15 Hz the spread is about
  twice as wide, as a discretisation error should be).  The taper lengths are made
  negligible (freq = 200 in the taper rule of optimization.c:364-365) since the misfit holds
  the tapered residual squared while the adjoint source carries the taper once.

The engine is bit-identical to the oracle's FP32 build (tests/test_oracle_golden.py and the GPU
parity tests), so these properties carry over to it.
"""
import numpy as np
import pytest

from fwiedu import models as M

NZ, NX, NT, DX, DT, PML, WATER = 60, 100, 700, 10.0, 0.001, 20, 15


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def model():
    vp = M.layered_model(NZ, NX, seed=3, water_rows=WATER, n_layers=4, n_anom=1)
    return vp, M.gardner(vp, water_rows=WATER)


@pytest.mark.parametrize("fs", [0, 1])
def test_reciprocity(port64, model, fs):
    vp, rho = model
    src = M.ricker(NT, DT, 15.0, 0.07)
    sv = M.line_survey(NZ, NX, DX, DX, DT, NT, 2, src, spacing_cells=40, first_cell=30, sdepth_cells=8,
                       gdepth_cells=8)
    shots = M.survey_shots(sv)
    assert shots[0].isx == 30 and shots[1].isx == 70 and shots[0].ix_min == 0
    tr, _ = port64.propagation(vp, rho, shots, DX, DX, DT, NT, PML, fs, 0.0, 2.0, 0, 0)
    a, b = tr[0][70], tr[1][30]  # source 30 -> receiver 70, source 70 -> receiver 30
    assert np.abs(a).max() > 1.0
    assert rel(a, b) < 5e-3  # measured 1.1e-3


def test_gradient_matches_finite_differences(port64, model):
    vp, rho = model
    src = M.ricker(NT, DT, 6.0, 0.12)
    sv = M.line_survey(NZ, NX, DX, DX, DT, NT, 3, src, spacing_cells=35, first_cell=15, sdepth_cells=2,
                       gdepth_cells=2)
    shots = M.survey_shots(sv)
    freq = 200.0
    obs, _ = port64.propagation(vp, rho, shots, DX, DX, DT, NT, PML, 1, 0.0, 2.0, 0, 0)
    vp0 = M.smooth_model(vp, 6.0, water_rows=WATER)
    _, g = port64.propagation(vp0, rho, shots, DX, DX, DT, NT, PML, 1, freq, 2.0, 0, 1, obs=obs)
    g = g.astype(np.float64)
    s0 = 1.0 / vp0.astype(np.float64)

    def misfit(s):
        res, _ = port64.propagation((1.0 / s).astype(np.float32), rho, shots, DX, DX, DT, NT, PML, 1, freq, 2.0, 0,
                                    2, obs=obs)
        return 0.5 * sum(float((np.asarray(r, np.float64) ** 2).sum()) for r in res)

    rng = np.random.default_rng(1)
    X, Z = np.meshgrid(np.arange(NX), np.arange(NZ), indexing="ij")
    ratios = []
    for _ in range(4):
        ds = np.zeros((NX, NZ))
        for _ in range(3):
            cx, cz = rng.uniform(15, NX - 15), rng.uniform(WATER + 8, NZ - 8)
            ds += rng.uniform(-1, 1) * np.exp(-((X - cx) ** 2 + (Z - cz) ** 2) / (2 * 6.0 ** 2))
        ds[:, :WATER + 2] = 0.0  # K at the sources and receivers unchanged
        ds *= 0.01 * s0.mean() / np.abs(ds).max()
        d1 = (misfit(s0 + 0.1 * ds) - misfit(s0 - 0.1 * ds)) / 0.2
        d2 = (misfit(s0 + 0.02 * ds) - misfit(s0 - 0.02 * ds)) / 0.04
        assert abs(d1 - d2) < 2e-3 * abs(d2)  # linear in the step
        gd = float((g * ds).sum())
        assert np.sign(gd) == np.sign(d2)
        ratios.append(gd / d2)
    ratios = np.array(ratios)
    assert np.all(np.abs(ratios / ratios.mean() - 1.0) < 0.2), ratios
