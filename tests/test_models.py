"""Seeded synthetic workloads: the layered model, Gardner density, wavelet, acquisition."""
import numpy as np

from fwiedu import models as M


def test_layered_model_properties():
    vp = M.layered_model(221, 601, seed=0)
    assert vp.shape == (601, 221) and vp.dtype == np.float32
    assert np.all(vp[:, :20] == 1500.0)
    body = vp[:, 20:]
    assert body.min() >= 1600.0 - 300.0 - 1 and body.max() <= 4500.0 + 300.0 + 1
    assert np.array_equal(vp, M.layered_model(221, 601, seed=0))
    assert not np.array_equal(vp, M.layered_model(221, 601, seed=1))


def test_gardner_and_smoothing():
    vp = M.layered_model(60, 80, seed=2, water_rows=5, anom_sigma=4)
    rho = M.gardner(vp, water_rows=5)
    assert np.all(rho[:, :5] == 1000.0)
    np.testing.assert_allclose(rho[:, 5:], 310.0 * vp[:, 5:].astype(np.float64) ** 0.25, rtol=1e-6)
    sm = M.smooth_model(vp, 3.0, water_rows=5)
    assert np.array_equal(sm[:, :5], vp[:, :5])
    assert np.abs(np.diff(sm[:, 10:], axis=1)).max() < np.abs(np.diff(vp[:, 10:], axis=1)).max()


def test_ricker_peak_frequency():
    src = M.ricker(4001, 0.001, 10.0, 0.15)
    assert abs(M.peak_frequency(src, 4001, 0.001) - 10.0) < 0.3
    assert int(np.argmax(np.abs(src))) == 150


def test_survey_and_windows():
    src = M.ricker(4001, 0.001)
    sv = M.line_survey(221, 601, 12.5, 12.5, 0.001, 4001, 60, src, spacing_cells=12, first_cell=0)
    assert sv.nshot == 60 and "reduced spacing" in sv.rule  # 59*12 > 600: spacing reduced to fit
    assert 0 <= min(sv.sx) and max(sv.sx) <= 600
    shots = M.survey_shots(sv)
    assert all(s.ix_min == 0 and s.ix_max == 600 for s in shots)  # receivers span the model
    assert shots[0].dtr == 12.5 and shots[0].ns == 4001
    sv2 = M.line_survey(50, 200, 10.0, 10.0, 0.001, 100, 1, src[:100], spacing_cells=5, first_cell=100)
    sv2.gx[0] = np.arange(120, 140, dtype=np.int32)
    s = M.survey_shots(sv2)[0]
    assert (s.ix_min, s.ix_max) == (90, 169) and s.isx == 10 and s.igx[0] == 30
