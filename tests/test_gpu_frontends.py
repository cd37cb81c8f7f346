"""The reference's own C front-ends as a user would link them against this library.

acoustic2d_modeling.c and acoustic2d_fwi.c, with the reference's parameter parsing, model and
wavelet readers, acquisition geometry and SU trace I/O (common, observation, dataio, cJSON),
are compiled unmodified and linked once against the reference's CPU engine
(oracle/_ref/acoustic2d_*_strict.exe) and once against libfwi_b200.so in place of
propagation/checkpoint/optimization (oracle/_ref/acoustic2d_*_b200.exe, `make -C oracle
frontends_b200`).  Both run on the same small synthetic inputs: the modeling output files must
be identical byte for byte, the FWI outputs (models, gradients, misfit history) within the
stated tolerances -- bit-exact engine arithmetic; FP64 sums in another order; FFT filters as
GEMMs.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from fwiedu import models as M

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "oracle", "_ref")
EXE = {(k, v): os.path.join(REF, f"acoustic2d_{k}_{v}.exe") for k in ("modeling", "fwi") for v in ("strict", "b200")}

NZ, NX, NT, DX, DT = 36, 64, 400, 10.0, 0.001
COMMON = dict(nx=NX, nz=NZ, nt=NT, dx=DX, dz=DX, dt=DT, freesurface=1, pmlThick=10, rhofile="", waterdepth=4,
              vp_water=1500.0, rho_water=1000.0, Gardner=1, Nshot=3, verbose=0)


def need_exes():
    missing = [p for p in EXE.values() if not os.path.exists(p)]
    if missing:
        pytest.skip("front-end executables not built (make -C oracle ref frontends_b200): " + ", ".join(missing))


def run(exe, cwd, **params):
    env = dict(os.environ, OMP_NUM_THREADS="1")
    args = [exe] + [f"{k}={v}" for k, v in params.items()]
    p = subprocess.run(args, cwd=cwd, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, f"{os.path.basename(exe)} failed:\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}"
    return p


def inputs(tmp):
    vp = M.layered_model(NZ, NX, seed=5, water_rows=4, anom_sigma=4)
    vp0 = M.smooth_model(vp, 3.0, water_rows=4)
    paths = {}
    for name, a in (("vp", vp), ("vp0", vp0)):
        paths[name] = str(tmp / f"{name}.bin")
        np.ascontiguousarray(a, np.float32).tofile(paths[name])  # [nx][nz]: column-major nz x nx
    paths["src"] = str(tmp / "ricker.bin")
    M.ricker(NT, DT, 12.0, 0.08).astype(np.float32).tofile(paths["src"])
    return paths


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def model_both(tmp, paths, **geom):
    out = {}
    for v in ("strict", "b200"):
        d = tmp / f"model_{v}"
        d.mkdir()
        run(EXE[("modeling", v)], d, srcfile=paths["src"], vpfile=paths["vp"], **COMMON, **geom)
        out[v] = sorted(glob.glob(str(d / "shots_p_*.su")))
    return out


def test_modeling_front_end_identical_output(tmp_path):
    need_exes()
    paths = inputs(tmp_path)
    geom = dict(fsx=4, ds=25, sdepth=2, offsmin=0, offsmax=NX - 1, dtr=1, gdepth=2, sampleRate=1)
    out = model_both(tmp_path, paths, **geom)
    assert out["strict"] and len(out["strict"]) == len(out["b200"])
    for a, b in zip(out["strict"], out["b200"]):
        assert os.path.basename(a) == os.path.basename(b)
        assert open(a, "rb").read() == open(b, "rb").read(), os.path.basename(a)


@pytest.mark.parametrize("sched", [dict(freq="10", filter="2", iteration="2", rx="1", rz="1"),
                                   dict(freq="6,10", filter="0,2", iteration="1,1", rx="2,1", rz="2,1")],
                         ids=["filter2", "multiscale_filter0"])
def test_fwi_front_end_matches_reference(tmp_path, sched):
    need_exes()
    paths = inputs(tmp_path)
    geom = dict(fsx=4, ds=25, sdepth=2, offsmin=0, offsmax=NX - 1, dtr=1, gdepth=2, sampleRate=1)
    record = model_both(tmp_path, paths, **geom)["strict"][0]
    res = {}
    for v in ("strict", "b200"):
        d = tmp_path / f"fwi_{v}"
        d.mkdir()
        params = dict(COMMON, verbose=1, srcfile=paths["src"], vpfile=paths["vp0"], recordfile=record, vpmin=1500.0,
                      vpmax=4700.0, rhomin=1000.0, rhomax=2700.0, precondition=1, **sched)
        run(EXE[("fwi", v)], d, **params)
        res[v] = d
    fft = "0" in sched["filter"]
    tol_model, tol_grad = (1e-5, 1e-4) if fft else (1e-6, 1e-6)
    niter = sum(int(x) for x in sched["iteration"].split(","))
    # verbose = 1: the same set of files as the reference writes, the engine's intermediate
    # files (propagation.c:917-944, 996-1005) included
    assert sorted(os.listdir(res["strict"])) == sorted(os.listdir(res["b200"]))
    for pattern, tol in (("vp_inversion_*.bin", tol_model), ("rho_inversion_*.bin", tol_model),
                         (f"objective_function_{niter:03d}.bin", tol_model), ("grad_iter*.bin", tol_grad),
                         ("vp_iter*.bin", tol_model), ("predicted_iter*_shot*.bin", tol_model),
                         ("adjsource_iter*_shot*.bin", tol_grad), ("gradient_raw_iter*_shot*.bin", tol_grad),
                         ("gradient_raw_iter???_*_*.bin", tol_grad), ("precond_iter*.bin", tol_grad)):
        fa = sorted(glob.glob(str(res["strict"] / pattern)))
        fb = sorted(glob.glob(str(res["b200"] / pattern)))
        assert fa and [os.path.basename(x) for x in fa] == [os.path.basename(x) for x in fb], pattern
        for a, b in zip(fa, fb):
            x, y = np.fromfile(b, np.float32), np.fromfile(a, np.float32)
            assert x.shape == y.shape and np.isfinite(x).all()
            assert rel(x, y) <= tol, f"{os.path.basename(a)}: rel {rel(x, y):.2e}"
            if not fft and "shot" in os.path.basename(a):
                # the first iteration's per-shot files come from the same model: bit for bit
                if "_iter001_" in os.path.basename(a):
                    assert np.array_equal(x, y), os.path.basename(a)


def test_snapshots_match_reference(tmp_path):
    """verbose = 2: wavefield snapshots every snapInterval steps (propagation.c:597-601, 717-723) --
    forward fields of the modeling and gradient passes, the reconstructed forward field and the
    adjoint field of the adjoint pass, with every free-surface row mirrored (the rows the
    stencil never reads again included) -- identical to the reference's files, bit for bit."""
    need_exes()
    paths = inputs(tmp_path)
    geom = dict(fsx=4, ds=25, sdepth=2, offsmin=0, offsmax=NX - 1, dtr=1, gdepth=2, sampleRate=1)
    record = model_both(tmp_path, paths, **geom)["strict"][0]
    env = dict(os.environ, snapInterval="100", shotInterval="2")
    res = {}
    for v in ("strict", "b200"):
        d = tmp_path / f"snap_{v}"
        d.mkdir()
        params = dict(COMMON, verbose=2, srcfile=paths["src"], vpfile=paths["vp0"], recordfile=record, vpmin=1500.0,
                      vpmax=4700.0, rhomin=1000.0, rhomax=2700.0, precondition=1, freq="10", filter="2",
                      iteration="1", rx="1", rz="1", **geom)
        args = [EXE[("fwi", v)]] + [f"{k}={val}" for k, val in params.items()]
        p = subprocess.run(args, cwd=d, env=dict(env, OMP_NUM_THREADS="1"), capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        res[v] = d
    names = sorted(os.listdir(res["strict"]))
    assert names == sorted(os.listdir(res["b200"]))
    snaps = [n for n in names if n.startswith("wavefield_")]
    kinds = {n.split("_iter")[0] for n in snaps}
    assert kinds == {"wavefield_forward", "wavefield_forward_reconstruction", "wavefield_backward"}, kinds
    for n in snaps:
        a = np.fromfile(res["strict"] / n, np.float32)
        b = np.fromfile(res["b200"] / n, np.float32)
        assert a.shape == b.shape and np.array_equal(a, b), f"{n}: rel {rel(b, a):.2e}"
