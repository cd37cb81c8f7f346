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
        files = sorted(os.listdir(df))
        obj = np.fromfile(os.path.join(df, [f for f in files if f.startswith("objective_function_")][0]), np.float32)
        grad1 = np.fromfile(os.path.join(df, [f for f in files if f.startswith("grad_iter001_")][0]), np.float32)
        vpinv = np.fromfile(os.path.join(df, [f for f in files if f.startswith("vp_inversion_")][0]), np.float32)
    np.savez_compressed(os.path.join(HERE, "demo_marm.npz"), inputs_sha256=digest(vp, vp0, src, geometry),
                        su_name=su, su_sha256=su_sha, modeling_files=np.array(mfiles),
                        fwi_files=np.array(files), objective=obj, grad_iter001=grad1, vp_inversion=vpinv)
    print(f"demo_marm.npz: {su} ({su_sha[:12]}), {len(files)} FWI files, objective {obj}")


if __name__ == "__main__":
    main()
