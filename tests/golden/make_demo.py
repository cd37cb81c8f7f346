"""Expected outputs of the demo-shaped front-end runs (tests/test_gpu_demo.py), from the reference.

The reference's Marmousi-II demo (demo/marm-ii/modeling.sh and fwi.sh) runs its two front-ends
with JSON acquisition geometry, a 30-cell absorbing layer, nt = 6001 at 1 ms, records
decimated by sampleRate = 2, a 36-cell water layer (1500 m/s, 1010 kg/m^3, Gardner density)
and verbose output.  The test runs the same front-ends with those parameters on a stated subset:
two shots of the demo's acquisition rule (shot k at x = 250 (k - 1) m, 25 m deep, 601 receivers
every 12.5 m at 25 m) written as an acquisition JSON, and a two-stage schedule (2 Hz with the
low-pass residual filter and 2-cell smoothing, then 10 Hz unfiltered) of one iteration each.
The model is a seeded synthetic stand-in of the demo's grid (221 x 601 at 12.5 m), not the
Marmousi-II file itself.

This script generates the inputs (deterministically; the test regenerates them and checks their
digest), runs the unmodified reference front-ends built in place
(oracle/_ref/acoustic2d_{modeling,fwi}_strict.exe, `make -C oracle ref`), and stores what the test
compares into demo_marm.npz: the digest of the inputs, the SHA-256 of the modeling SU file, the
files each front-end writes, the misfit history, the first iteration's gradient and the final model.

It also runs the reference's FWI front-end a second time, linked with a single-precision build of
the FFT library shim (acoustic2d_fwi_strict_f32fft.exe; the transforms round as an FFTW float build
does), on the same observed data, and stores how far each compared output moves
(`fft_sensitivity`: relative L2 change of the gradient and final model, largest relative change of
the misfits).  These are the reference's own precision for this run: its low-pass filtered 2 Hz
stage forms the gradient from a residual that barely overlaps the 10 Hz wavelet's band, and the
first iteration's gradient moves by ~1.4e-4 when only the FFT's rounding changes, while the
predicted data and the pseudo-Hessian stay bit-identical.

    python tests/golden/make_demo.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "fwi-edu_b200"))

from fwiedu import models as M  # noqa: E402

NZ, NX, NT, D, DT, PML = 221, 601, 6001, 12.5, 0.001, 30
WATER = 36
SHOT_IDS = (1, 16)
COMMON = dict(nx=NX, nz=NZ, nt=NT, dx=D, dz=D, dt=DT, freesurface=1, pmlThick=PML, rhofile="", waterdepth=WATER,
              vp_water=1500.0, rho_water=1010.0, Gardner=1, verbose=1)
MODELING = dict(Nshot=len(SHOT_IDS), fsx=0, ds=20, sdepth=2, offsmin=0, offsmax=600, dtr=1, gdepth=2, sampleRate=2)
FWI = dict(Nshot=len(SHOT_IDS), vpmin=1500, vpmax=4700, rhomin=1000, rhomax=2700, precondition=1, freq="2,10",
           filter="0,2", iteration="1,1", rx="2,1", rz="2,1")
ENV = dict(shotInterval="1", snapInterval="1000")


def inputs():
    """The stand-in model (true and smoothed starting model), the wavelet and the JSON geometry."""
    vp = M.layered_model(NZ, NX, seed=2024, water_rows=WATER)
    vp0 = M.smooth_model(vp, 10.0, water_rows=WATER)
    src = M.ricker(NT, DT, 10.0, 0.15)
    rec = []
    for sid in SHOT_IDS:
        gx = [12.5 * i for i in range(NX)]
        rec.append({"shotID": sid, "sx": 250.0 * (sid - 1), "sz": 25.0, "ntr": NX, "gx": gx, "gz": [25.0] * NX})
    geometry = {"model": {"nx": NX, "nz": NZ, "dx": D, "dz": D}, "record": rec,
                "acquisition": {"type": "surface", "note": "two shots of the demo's rule"}}
    return vp, vp0, src, geometry


def digest(vp, vp0, src, geometry):
    h = hashlib.sha256()
    for a in (vp, vp0, src):
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    h.update(json.dumps(geometry, sort_keys=True).encode())
    return h.hexdigest()


def write_inputs(d, vp, vp0, src, geometry):
    paths = {"vp": os.path.join(d, "vp.bin"), "vp0": os.path.join(d, "vp0.bin"), "src": os.path.join(d, "src.bin"),
             "json": os.path.join(d, "acquisition.json")}
    np.ascontiguousarray(vp, np.float32).tofile(paths["vp"])
    np.ascontiguousarray(vp0, np.float32).tofile(paths["vp0"])
    np.ascontiguousarray(src, np.float32).tofile(paths["src"])
    with open(paths["json"], "w") as f:
        json.dump(geometry, f)
    return paths


def run(exe, cwd, threads=None, **params):
    env = dict(os.environ, **ENV)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    args = [exe] + [f"{k}={v}" for k, v in params.items()]
    p = subprocess.run(args, cwd=cwd, env=env, capture_output=True, text=True, timeout=3600)
    if p.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} failed:\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    return p


def run_demo(modeling_exe, fwi_exe, workdir, paths, threads=None):
    """Both front-ends in workdir/modeling and workdir/fwi; returns the two directories."""
    dm, df = os.path.join(workdir, "modeling"), os.path.join(workdir, "fwi")
    os.makedirs(dm)
    os.makedirs(df)
    run(modeling_exe, dm, threads, srcfile=paths["src"], vpfile=paths["vp"], jsonfile=paths["json"], **COMMON,
        **MODELING)
    su = [f for f in os.listdir(dm) if f.startswith("shots_p_") and f.endswith(".su")]
    assert len(su) == 1, su
    run(fwi_exe, df, threads, srcfile=paths["src"], vpfile=paths["vp0"], recordfile=os.path.join(dm, su[0]),
        **COMMON, **FWI)
    return dm, df


def outputs(df):
    """misfit history, first iteration's gradient, final model of an FWI run directory"""
    files = sorted(os.listdir(df))

    def load(prefix):
        return np.fromfile(os.path.join(df, [f for f in files if f.startswith(prefix)][0]), np.float32)

    return files, load("objective_function_"), load("grad_iter001_"), load("vp_inversion_")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def main():
    ref = os.path.join(ROOT, "oracle", "_ref")
    vp, vp0, src, geometry = inputs()
    with tempfile.TemporaryDirectory() as t:
        paths = write_inputs(t, vp, vp0, src, geometry)
        dm, df = run_demo(os.path.join(ref, "acoustic2d_modeling_strict.exe"),
                          os.path.join(ref, "acoustic2d_fwi_strict.exe"), t, paths, threads=os.cpu_count())
        su = [f for f in os.listdir(dm) if f.endswith(".su")][0]
        su_sha = hashlib.sha256(open(os.path.join(dm, su), "rb").read()).hexdigest()
        mfiles = sorted(os.listdir(dm))
        files, obj, grad1, vpinv = outputs(df)
        # the same FWI run on the single-precision FFT build, same observed data
        df2 = os.path.join(t, "fwi_f32fft")
        os.makedirs(df2)
        run(os.path.join(ref, "acoustic2d_fwi_strict_f32fft.exe"), df2, os.cpu_count(), srcfile=paths["src"],
            vpfile=paths["vp0"], recordfile=os.path.join(dm, su), **COMMON, **FWI)
        _, obj2, grad2, vpinv2 = outputs(df2)
    sens = np.array([rel(grad2, grad1), rel(vpinv2, vpinv), float(np.max(np.abs(obj2 - obj) / np.abs(obj)))])
    np.savez_compressed(os.path.join(HERE, "demo_marm.npz"), inputs_sha256=digest(vp, vp0, src, geometry),
                        su_name=su, su_sha256=su_sha, modeling_files=np.array(mfiles),
                        fwi_files=np.array(files), objective=obj, grad_iter001=grad1, vp_inversion=vpinv,
                        fft_sensitivity=sens)
    print(f"demo_marm.npz: {su} ({su_sha[:12]}), {len(files)} FWI files, objective {obj}; "
          f"reference's FFT-rounding sensitivity: gradient {sens[0]:.3e}, model {sens[1]:.3e}, misfit {sens[2]:.3e}")


if __name__ == "__main__":
    main()
