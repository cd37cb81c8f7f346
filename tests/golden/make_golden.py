"""Generate the golden vectors of tests/golden/ by running the reference itself.

The FWI-EDU C sources are compiled unmodified from the reference checkout against
the SU/FFTW shim (``make -C oracle ref``; strict IEEE build, OpenMP at one thread so
its reductions run in sequential order).  This script drives the reference's own
public entry points (iso_acoustic2d_propagation, calculate_objective_value,
calculate_step_length, compute_model_perturbation, smooth2D,
calculate_peak_frequency) on small seeded cases and stores inputs and outputs as
compressed .npz files.  The reference checkout is needed only here; the fixtures
travel with the repository.

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "fwi-edu_b200"))
os.environ.setdefault("OMP_NUM_THREADS", "1")

import numpy as np  # noqa: E402

import pyoracle as po  # noqa: E402
from fwiedu import models as M  # noqa: E402

DX = 12.5


def geometry(nz, nx, nt, dt, nshot, seed, f=12.0, t0=0.08, narrow=True, src_depth=1, rec_depth=1, dup=False):
    src = M.ricker(nt, dt, f, t0)
    sv = M.line_survey(nz, nx, DX, DX, dt, nt, nshot, src, spacing_cells=nx // (nshot + 1), first_cell=5,
                       sdepth_cells=src_depth, gdepth_cells=rec_depth)
    if narrow and nshot > 1:  # a shot whose receivers do not span the model: window and quirk of the global vp index
        sv.gx[1] = np.arange(nx // 4, 3 * nx // 4, dtype=np.int32)
        sv.gz[1] = np.full(len(sv.gx[1]), rec_depth + 1, np.int32)
    if dup:  # two receivers on the same cell, and one on the free-surface row
        sv.gx[0] = np.concatenate([sv.gx[0], sv.gx[0][[7, 7]]]).astype(np.int32)
        sv.gz[0] = np.concatenate([sv.gz[0], np.array([0, rec_depth], np.int32)]).astype(np.int32)
    return M.survey_shots(sv)


def pack_shots(shots):
    d = {}
    d["shot_scalars"] = np.array([[s.shotID, s.isx, s.isz, s.ns, s.sampleRate, s.ix_min, s.ix_max] for s in shots], np.int32)
    d["shot_floats"] = np.array([[s.dt, s.dtr, s.fpeak, s.sx, s.sz] for s in shots], np.float32)
    d["src"] = np.asarray(shots[0].src, np.float32)
    for i, s in enumerate(shots):
        d[f"igx{i}"] = np.asarray(s.igx, np.int32)
        d[f"igz{i}"] = np.asarray(s.igz, np.int32)
    return d


def case(name, nz, nx, nt, dt, pml, fs, nshot, seed, problems=(0, 1, 2), precondition=1, sr=1, obs_src_depth=None,
         filt=2.0, **kw):
    ref = po.Reference("strict")
    vp = M.layered_model(nz, nx, seed=seed, water_rows=6, anom_sigma=4)
    rho = M.gardner(vp, water_rows=6)
    shots = geometry(nz, nx, nt, dt, nshot, seed, **kw)
    if sr > 1:
        for s in shots:
            s.sampleRate = sr
            s.ns = (nt - 1) // sr + 1
            s.dt = float(np.float32(np.float32(dt) * sr))
    out = dict(vp=vp, rho=rho, nz=nz, nx=nx, nt=nt, dt=np.float32(dt), dx=np.float32(DX), pml=pml, fs=fs,
               precondition=precondition, nshot=nshot, filter=np.float32(filt))
    out.update(pack_shots(shots))
    out["fpeak_ref"] = np.float32(ref.peak_frequency(shots[0].src, nt, dt))
    obs_shots = shots
    if obs_src_depth is not None:  # observed data from another source depth than the modelled one
        kw2 = dict(kw)
        kw2["src_depth"] = obs_src_depth
        obs_shots = geometry(nz, nx, nt, dt, nshot, seed, **kw2)
    obs, _ = ref.propagation(vp, rho, obs_shots, DX, DX, dt, nt, pml, fs, 0.0, 2.0, precondition, 0)
    for i, t in enumerate(obs):
        out[f"obs{i}"] = t
    if 1 in problems:
        vp0 = M.smooth_model(vp, 3.0, water_rows=6)
        rho0 = M.gardner(vp0, water_rows=6)
        out["vp0"], out["rho0"] = vp0, rho0
        freq = 10.0
        adj, grad = ref.propagation(vp0, rho0, shots, DX, DX, dt, nt, pml, fs, freq, filt, precondition, 1, obs=obs)
        for i, t in enumerate(adj):
            out[f"adj{i}"] = t
        out["grad"] = grad
        out["fun1"] = np.float32(ref.objective(adj, shots))
        # the line-search step of acoustic2d_fwi.c:418-449 with rx = rz = 1
        sm = ref.smooth2d(grad, 1, 1)
        sm = ref.smooth2d(sm, 1, 0)
        out["grad_smooth"] = sm
        slow = (1.0 / vp0).astype(np.float32)
        scalar, perturb = ref.model_perturbation(0.01, slow, sm)
        out["pert_scalar"] = np.float32(scalar)
        out["perturb"] = perturb
        vp1 = 1.0 / (slow + perturb)
        vp1 = np.clip(vp1.astype(np.float32), 1500.0, 4700.0).astype(np.float32)
        vp1[:, :6] = 1500.0
        rho1 = M.gardner(vp1, water_rows=6)
        out["vp1"], out["rho1"] = vp1, rho1
        if 2 in problems:
            res, _ = ref.propagation(vp1, rho1, shots, DX, DX, dt, nt, pml, fs, freq, filt, precondition, 2, obs=obs)
            for i, t in enumerate(res):
                out[f"res{i}"] = t
            out["fun2"] = np.float32(ref.objective(res, shots))
            out["steplen"] = np.float32(ref.step_length(adj, res, shots))
        # a wider smoothing window exercises the weights and the edge handling
        out["grad_smooth3"] = ref.smooth2d(ref.smooth2d(grad, 3, 1), 2, 0)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {os.path.getsize(path) / 1024:.0f} KiB")


def wavenumber_case():
    """lowpass2d / bandpass2d (common.c:1042-1284, defined but not called by the reference's
    engine) on a seeded gradient-like field; the reference tapers its input in place, which
    the fixture records as well."""
    import ctypes as C
    ref = po.Reference("strict")
    L = ref.lib
    nz, nx, dz, dx = 40, 70, 12.5, 10.0
    rng = np.random.default_rng(13)
    base = M.smooth_model(rng.standard_normal((nx, nz)).astype(np.float32) * 100.0 + 2000.0, 2.0).astype(np.float32)
    out = dict(field=base, nz=nz, nx=nx, dz=np.float32(dz), dx=np.float32(dx))
    for name, fn, kpass, kcut in (("low", L.lowpass2d, 0.02, 0.04), ("band", L.bandpass2d, 0.015, 0.035)):
        s = base.copy()
        y = np.zeros_like(s)
        fn(po.rows(s), nz, nx, C.c_float(dz), C.c_float(dx), C.c_float(kpass), C.c_float(kcut), po.rows(y))
        out[f"{name}_kpass"] = np.float32(kpass)
        out[f"{name}_kcut"] = np.float32(kcut)
        out[f"{name}_out"] = y
        out[f"{name}_tapered_input"] = s
    path = os.path.join(HERE, "aux_wavenumber.npz")
    np.savez_compressed(path, **out)
    print(f"aux_wavenumber: {os.path.getsize(path) / 1024:.0f} KiB")


def main():
    if not po.ref_available("strict"):
        if not po.build_ref():
            raise SystemExit("the reference checkout is needed to regenerate the golden vectors")
    only = set(sys.argv[1:])
    if only:  # regenerate the named cases only
        global case
        full = case
        case = lambda name, *a, **k: full(name, *a, **k) if name in only else None  # noqa: E731
    case("fs1_small", 40, 70, 300, 0.001, 8, 1, 3, seed=3)
    case("fs0_small", 40, 70, 300, 0.001, 8, 0, 3, seed=4)
    # nt = 200 gives d = 20 with nt % d == 0: the last segment replays d-1 steps
    case("fs1_ntmod", 33, 48, 200, 0.001, 6, 1, 2, seed=5)
    # receivers on the free-surface row and on one shared cell; source ON the free-surface row,
    # where the forward pass loses the source and the replay keeps it (propagation.c:558-564 vs
    # :656-662).  The forward field is then zero, so the pseudo-Hessian is zero and the reference's
    # per-shot preconditioner divides 0 by 0: this case runs without preconditioning.
    case("fs1_edges", 36, 52, 240, 0.001, 5, 1, 2, seed=6, dup=True, src_depth=0, obs_src_depth=1, precondition=0)
    case("noprec", 36, 60, 220, 0.001, 7, 1, 2, seed=7, precondition=0)
    case("sr2_fwd", 36, 60, 301, 0.001, 7, 1, 2, seed=8, problems=(0,), sr=2)
    # FFT residual filters (optimization.c:368-415): lowpass and bandpass in time and space
    case("filt0", 40, 70, 300, 0.001, 8, 1, 3, seed=9, filt=0.0)
    case("filt1", 40, 70, 300, 0.001, 8, 1, 2, seed=10, problems=(0, 1), filt=1.0)
    # observed data every 2nd step: the adjoint source is interpolated back to every step
    # (interpolate_traces, common.c:482-582), with and without the lowpass
    case("sr2_grad", 36, 60, 301, 0.001, 7, 1, 2, seed=11, sr=2)
    case("sr2_filt0", 36, 60, 301, 0.001, 7, 1, 2, seed=12, problems=(0, 1), sr=2, filt=0.0)
    if not only or "wavenumber" in only:
        wavenumber_case()


if __name__ == "__main__":
    main()
