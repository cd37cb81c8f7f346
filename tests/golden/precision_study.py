"""Precision study of the checkpoint snapshots on the large grid (1201 x 4001 at 5 m, 20 Hz
Ricker, dt = 0.4 ms, nt = 8001, 40-cell absorbing layer, free surface, 4001 receivers): may the
snapshots the replay restarts from and the imaging reads be stored in FP16 or BF16, each with
its own max-abs scale?  Only where the gradient tolerance (1e-4 relative) still holds.

Stated fraction: one shot of the 100-shot survey (the middle one), run with the oracle's C
restatement of the engine (oracle/libfwi_oracle_f32.so, bit-exact with the reference and the
CUDA engine in FP32) and its FP64 build (libfwi_oracle_f64.so) as the error reference.  For each
snapshot format: the gradient (problem 1) and one line-search step as acoustic2d_fwi.c:418-465
takes it (smoothing, histogram-scaled perturbation, trial model, problem 2, step length);
errors of the seismogram, the adjoint source, the gradient and the step length against the FP64
build.  Observed data: the FP64 forward of the true model.  Writes precision_config3.json beside
this script.

    OMP_NUM_THREADS=<cores> python tests/golden/precision_study.py
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "fwi-edu_b200"))

import pyoracle as po  # noqa: E402
from fwiedu import models as M  # noqa: E402

NZ, NX, D, DT, NT, PML, FS, WATER = 1201, 4001, 5.0, 0.0004, 8001, 40, 1, 20
P = dict(rx=1, rz=1, waterdepth=WATER, vp_water=1500.0, rho_water=1000.0, vpmin=1500.0, vpmax=4700.0,
         rhomin=1000.0, rhomax=2700.0)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def iteration(port, vp0, rho0, shots, obs):
    """gradient + one line-search step of the FWI loop (acoustic2d_fwi.c:411-465), FP32 model ops"""
    adj, g = port.propagation(vp0, rho0, shots, D, D, DT, NT, PML, FS, 20.0, 2.0, 1, 1, obs=obs)
    g = np.asarray(g, np.float32)
    slow = np.where(vp0 != 0, 1.0 / vp0, 0).astype(np.float32)
    p32 = po.Port(32)
    gs = p32.smooth2d(p32.smooth2d(g, P["rz"], 1), P["rx"], 0)
    _, pert = p32.model_perturbation(0.01, slow, gs)
    vpt, rhot = p32.fwi_trial(slow, pert, P["waterdepth"], P["vp_water"], P["rho_water"], P["vpmin"], P["vpmax"],
                              P["rhomin"], P["rhomax"])
    res, _ = port.propagation(vpt, rhot, shots, D, D, DT, NT, PML, FS, 20.0, 2.0, 1, 2, obs=obs)
    steplen = p32.step_length([np.asarray(a, np.float32) for a in adj], [np.asarray(r, np.float32) for r in res])
    return adj, g, steplen


def main():
    t0 = time.time()
    vp = M.layered_model(NZ, NX, seed=7, water_rows=WATER)
    rho = M.gardner(vp, water_rows=WATER)
    vp0 = M.smooth_model(vp, 15.0, water_rows=WATER)
    rho0 = M.gardner(vp0, water_rows=WATER)
    src = M.ricker(NT, DT, 20.0, 0.075)
    sv = M.line_survey(NZ, NX, D, D, DT, NT, 100, src, spacing_cells=(NX - 1) // 100, first_cell=0)
    shots = [M.survey_shots(sv)[50]]
    p64, p32 = po.Port(64), po.Port(32)
    obs64, _ = p64.propagation(vp, rho, shots, D, D, DT, NT, PML, FS, 0.0, 2.0, 1, 0)
    obs = [np.asarray(o, np.float32) for o in obs64]
    obs32, _ = p32.propagation(vp, rho, shots, D, D, DT, NT, PML, FS, 0.0, 2.0, 1, 0)
    out = {"grid": f"{NZ}x{NX} at {D} m, nt {NT}, dt {DT} s, 20 Hz Ricker, pml {PML}, free surface",
           "sample": f"1 shot (ix = {shots[0].isx + shots[0].ix_min}) of the 100-shot survey, "
                     f"{len(shots[0].igx)} receivers",
           "reference": "FP64 build of the same algorithm (oracle/libfwi_oracle_f64.so)",
           "seismogram_fp32_rel_l2": rel(obs32[0], obs64[0])}
    print("seismogram", out["seismogram_fp32_rel_l2"], flush=True)
    adj64, g64, s64 = iteration(p64, vp0, rho0, shots, obs)
    out["steplen_fp64"] = s64
    for mode, label in ((0, "fp32"), (1, "fp16_maxabs"), (2, "bf16")):
        p32.set_checkpoint_precision(mode)
        try:
            adj, g, s = iteration(p32, vp0, rho0, shots, obs)
        finally:
            p32.set_checkpoint_precision(0)
        out[label] = {"adjoint_source_rel_l2": rel(adj[0], adj64[0]), "gradient_rel_l2": rel(g, g64),
                      "steplen": s, "steplen_rel": abs(s - s64) / abs(s64)}
        print(label, out[label], flush=True)
    out["gradient_tolerance"] = 1e-4
    out["cpu_seconds"] = time.time() - t0
    with open(os.path.join(HERE, "precision_config3.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
