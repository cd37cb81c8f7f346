"""ctypes bindings to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:

* the port -- this project's C restatement (fwi_oracle.c), built as
  ``libfwi_oracle_f32.so`` (bit-exact FP32) and ``libfwi_oracle_f64.so`` (FP64 build of
  the same algorithm);
* the reference itself -- the unmodified FWI-EDU C sources compiled against the SU/FFTW
  shim into ``oracle/_ref/libfwiref_*.so`` (present only where the reference checkout
  was available at build time; the built library travels with the repository snapshot).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
Shot objects are duck-typed: any object with the attributes of ``fwiedu.models.Shot``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# the reference checkout (C implementation); FWI_REFERENCE_ROOT overrides the default location
REFERENCE_ROOT = os.environ.get("FWI_REFERENCE_ROOT", "/root/reference/FWILab2d/FWILab2dCLangV1.2.6")

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_fpp = C.POINTER(_fp)


class OrcShot(C.Structure):
    _fields_ = [("shotID", C.c_int), ("isx", C.c_int), ("isz", C.c_int), ("ntr", C.c_int),
                ("ns", C.c_int), ("sampleRate", C.c_int), ("ix_min", C.c_int), ("ix_max", C.c_int),
                ("dt", C.c_float), ("dtr", C.c_float), ("fpeak", C.c_float),
                ("src", _fp), ("igx", _ip), ("igz", _ip)]


class Record2D(C.Structure):
    """The reference's shot record (observation.h:18-48)."""
    _fields_ = [("shotID", C.c_int), ("sx", C.c_float), ("sz", C.c_float), ("isx", C.c_int),
                ("isz", C.c_int), ("fpeak", C.c_float), ("src", _fp), ("gx", _fp), ("gz", _fp),
                ("igx", _ip), ("igz", _ip), ("sampleRate", C.c_int), ("ntr", C.c_int),
                ("ns", C.c_int), ("dtr", C.c_float), ("dt", C.c_float), ("ix_min", C.c_int),
                ("ix_max", C.c_int), ("traces_vx", _fpp), ("traces_vz", _fpp), ("traces_p", _fpp),
                ("precond", _fpp), ("grad", _fpp)]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a, t=_fp):
    return a.ctypes.data_as(t)


def rows(a: np.ndarray):
    """float** row-pointer view of a C-contiguous (n2, n1) float32 array (alloc2float layout)."""
    assert a.dtype == np.float32 and a.flags.c_contiguous
    n2 = a.shape[0]
    n1 = int(np.prod(a.shape[1:])) if a.ndim > 1 else 1
    arr = (_fp * max(n2, 1))()
    base = a.ctypes.data
    for i in range(n2):
        arr[i] = C.cast(base + i * n1 * 4, _fp)
    return arr


# ----------------------------------------------------------------------------- port
class Port:
    """The C restatement; ``precision`` 32 (bit-exact) or 64 (FP64 build)."""

    def __init__(self, precision: int = 32):
        name = "libfwi_oracle_f32.so" if precision == 32 else "libfwi_oracle_f64.so"
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            build_port()
        self.lib = C.CDLL(path)
        self.precision = precision
        L = self.lib
        L.orc_forward.restype = C.c_int
        L.orc_shot_gradient.restype = C.c_int
        L.orc_propagation.restype = C.c_int
        for f in ("orc_objective", "orc_step_length", "orc_model_perturbation"):
            getattr(L, f).restype = C.c_float
        self._keep = []

    def _shot(self, s):
        igx, igz, src = _i32(s.igx), _i32(s.igz), _f32(s.src)
        self._keep += [igx, igz, src]
        return OrcShot(s.shotID, s.isx, s.isz, len(igx), s.ns, s.sampleRate, s.ix_min, s.ix_max,
                       s.dt, s.dtr, s.fpeak, _ptr(src), _ptr(igx, _ip), _ptr(igz, _ip))

    def setup(self, vpm, rhom, pml, dx, dz, dt, fpeak):
        nx, nz = vpm.shape
        Nx, Nz = nx + 2 * pml, nz + 2 * pml
        dt_np = np.float32 if self.precision == 32 else np.float64
        outs = [np.zeros((Nx, Nz), dt_np) for _ in range(7)]
        self.lib.orc_setup(_ptr(_f32(vpm)), _ptr(_f32(rhom)), nz, nx, pml, C.c_float(dx), C.c_float(dz),
                           C.c_float(dt), C.c_float(fpeak), *[o.ctypes.data_as(C.c_void_p) for o in outs])
        return dict(zip(("coef1", "coef2", "coef3", "K", "invrho", "invrhox", "invrhoz"), outs))

    def forward(self, shot, vp, rho, dx, dz, dt, nt, pml, fs):
        """Forward modeling of one shot on the shot's window of the global model."""
        vpw = _f32(vp[shot.ix_min:shot.ix_max + 1])
        rhow = _f32(rho[shot.ix_min:shot.ix_max + 1])
        nxx, nz = vpw.shape
        tr = np.zeros((len(shot.igx), shot.ns), np.float32)
        rc = self.lib.orc_forward(C.byref(self._shot(shot)), _ptr(vpw), _ptr(rhow), nz, nxx, C.c_float(dx),
                                  C.c_float(dz), C.c_float(dt), nt, pml, fs, _ptr(tr))
        self._keep.clear()
        if rc:
            raise ValueError(f"orc_forward: status {rc}")
        return tr

    def shot_gradient(self, shot, vp, rho, dx, dz, dt, nt, pml, fs, freq, filt, precondition, obs):
        """One shot's gradient and preconditioner on its window (orc_shot_gradient, FP32 port):
        (adjoint source, g, h), g and h of shape (ix_max - ix_min + 1, nz)."""
        if self.precision != 32:
            raise ValueError("shot_gradient wraps the FP32 port")
        vp, rho = _f32(vp), _f32(rho)
        nx, nz = vp.shape
        nxx = shot.ix_max - shot.ix_min + 1
        pre = np.zeros((len(shot.igx), shot.ns), np.float32)
        g = np.zeros((nxx, nz), np.float32)
        h = np.zeros((nxx, nz), np.float32)
        rc = self.lib.orc_shot_gradient(C.byref(self._shot(shot)), _ptr(vp), _ptr(rho), nz, nx, C.c_float(dx),
                                        C.c_float(dz), C.c_float(dt), nt, pml, fs, C.c_float(freq), int(filt),
                                        precondition, _ptr(_f32(obs)), _ptr(pre), _ptr(g), _ptr(h))
        self._keep.clear()
        if rc:
            raise ValueError(f"orc_shot_gradient: status {rc}")
        return pre, g, h

    def set_checkpoint_precision(self, mode):
        """Checkpoint snapshots: 0 oracle precision, 1 FP16 with max-abs scaling, 2 BF16."""
        self.lib.orc_set_checkpoint_precision(int(mode))

    def global_precondition(self, grad, precond, alpha=0.005):
        """orc_global_precondition on float32 arrays, in place."""
        n = grad.size
        self.lib.orc_global_precondition(_ptr(grad), _ptr(precond), n, C.c_float(alpha))
        return grad

    def propagation(self, vp, rho, shots, dx, dz, dt, nt, pml, fs, freq, filt, precondition, problem,
                    obs=None, pre=None):
        """Mirror of iso_acoustic2d_propagation; returns (pre traces list, grad or None)."""
        vp, rho = _f32(vp), _f32(rho)
        nx, nz = vp.shape
        ns = len(shots)
        cs = (OrcShot * ns)(*[self._shot(s) for s in shots])
        pre = [np.zeros((len(s.igx), s.ns), np.float32) if pre is None else _f32(pre[i]).copy()
               for i, s in enumerate(shots)]
        obs = [np.zeros((len(s.igx), s.ns), np.float32) if obs is None else _f32(obs[i]) for i, s in enumerate(shots)]
        pp = (_fp * ns)(*[_ptr(p) for p in pre])
        op = (_fp * ns)(*[_ptr(o) for o in obs])
        grad = np.zeros((nx, nz), np.float32) if problem == 1 else None
        rc = self.lib.orc_propagation(_ptr(vp), _ptr(rho), cs, ns, nz, nx, C.c_float(dx), C.c_float(dz),
                                      C.c_float(dt), nt, pml, fs, C.c_float(freq), C.c_float(filt),
                                      precondition, problem, op, pp,
                                      _ptr(grad) if grad is not None else None)
        self._keep.clear()
        if rc:
            raise ValueError(f"orc_propagation: status {rc}")
        return pre, grad

    def objective(self, traces):
        tr = [_f32(t) for t in traces]
        p = (_fp * len(tr))(*[_ptr(t) for t in tr])
        ntr = _i32([t.shape[0] for t in tr]); ns = _i32([t.shape[1] for t in tr])
        return float(self.lib.orc_objective(p, _ptr(ntr, _ip), _ptr(ns, _ip), len(tr)))

    def step_length(self, pre0, pre1):
        a = [_f32(t) for t in pre0]; b = [_f32(t) for t in pre1]
        pa = (_fp * len(a))(*[_ptr(t) for t in a]); pb = (_fp * len(b))(*[_ptr(t) for t in b])
        ntr = _i32([t.shape[0] for t in a]); ns = _i32([t.shape[1] for t in a])
        return float(self.lib.orc_step_length(pa, pb, _ptr(ntr, _ip), _ptr(ns, _ip), len(a)))

    def model_perturbation(self, fraction, slow, grad):
        slow, grad = _f32(slow), _f32(grad)
        out = np.zeros_like(grad)
        s = self.lib.orc_model_perturbation(C.c_float(fraction), _ptr(slow), _ptr(grad), _ptr(out), grad.size)
        return float(s), out

    def smooth2d(self, a, N, zdir):
        a = _f32(a)
        out = np.zeros_like(a)
        nx, nz = a.shape
        self.lib.orc_smooth2d(_ptr(a), _ptr(out), nx, nz, N, zdir)
        return out

    def taper(self, tr, lt, lr):
        tr = _f32(tr).copy()
        ntr, nt = tr.shape
        self.lib.orc_taper_traces(_ptr(tr), nt, ntr, lt, lr)
        return tr

    def fwi_trial(self, slow, perturb, waterdepth, vp_water, rho_water, vpmin, vpmax, rhomin, rhomax, gardner=1):
        slow, perturb = _f32(slow), _f32(perturb)
        nx, nz = slow.shape
        vp = np.zeros_like(slow); rho = np.zeros_like(slow)
        self.lib.orc_fwi_trial(_ptr(slow), _ptr(perturb), _ptr(vp), _ptr(rho), nx, nz, waterdepth,
                               C.c_float(vp_water), C.c_float(rho_water), C.c_float(vpmin), C.c_float(vpmax),
                               C.c_float(rhomin), C.c_float(rhomax), gardner)
        return vp, rho

    def fwi_update(self, slow, vp, rho, perturb, steplen, waterdepth, vp_water, rho_water, vpmin, vpmax,
                   rhomin, rhomax, gardner=1):
        slow, vp, rho, perturb = _f32(slow).copy(), _f32(vp).copy(), _f32(rho).copy(), _f32(perturb)
        nx, nz = slow.shape
        self.lib.orc_fwi_update(_ptr(slow), _ptr(vp), _ptr(rho), _ptr(perturb), C.c_float(steplen), nx, nz,
                                waterdepth, C.c_float(vp_water), C.c_float(rho_water), C.c_float(vpmin),
                                C.c_float(vpmax), C.c_float(rhomin), C.c_float(rhomax), gardner)
        return slow, vp, rho

    def checkpoint_interval(self, nt):
        return int(self.lib.orc_checkpoint_interval(nt))

    def checkpoint_count(self, nt):
        return int(self.lib.orc_checkpoint_count(nt))


def build_port():
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)


# ------------------------------------------------------------------------ reference
def ref_available(flavor: str = "strict") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libfwiref_{flavor}.so"))


def build_ref():
    """Compile the unmodified reference sources against the shim (needs the reference checkout)."""
    if not os.path.isdir(REFERENCE_ROOT):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", "-j8", f"REFROOT={REFERENCE_ROOT}"], check=True)
    return True


def host_flavor() -> str:
    """The fast reference build that the current host CPU can execute."""
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        flags = ""
    v4 = all(f in flags for f in ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"))
    return "fast_v4" if v4 and ref_available("fast_v4") else "fast_v3"


class Reference:
    """The reference C library itself, driven through its own public entry point
    iso_acoustic2d_propagation (propagation.h:133-142) with Record2D shot records."""

    def __init__(self, flavor: str = "strict"):
        path = os.path.join(REF_DIR, f"libfwiref_{flavor}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.lib.calculate_peak_frequency.restype = C.c_float
        self.lib.calculate_peak_frequency.argtypes = [_fp, C.c_int, C.c_float]
        self.lib.calculate_objective_value.restype = C.c_float
        self.lib.calculate_step_length.restype = C.c_float
        self.lib.compute_model_perturbation.restype = C.c_float
        self._keep = []

    def _record(self, s, traces):
        igx, igz, src = _i32(s.igx), _i32(s.igz), _f32(s.src)
        gx = ((igx + s.ix_min).astype(np.float32) * np.float32(s.dtr)).astype(np.float32)
        gz = igz.astype(np.float32)
        rp = rows(traces)
        self._keep += [igx, igz, src, gx, gz, rp, traces]
        r = Record2D()
        r.shotID = s.shotID; r.sx = s.sx; r.sz = s.sz; r.isx = s.isx; r.isz = s.isz; r.fpeak = s.fpeak
        r.src = _ptr(src); r.gx = _ptr(gx); r.gz = _ptr(gz); r.igx = _ptr(igx, _ip); r.igz = _ptr(igz, _ip)
        r.sampleRate = s.sampleRate; r.ntr = len(igx); r.ns = s.ns; r.dtr = s.dtr; r.dt = s.dt
        r.ix_min = s.ix_min; r.ix_max = s.ix_max
        r.traces_p = C.cast(rp, _fpp)
        return r

    def peak_frequency(self, src, nt, dt):
        src = _f32(src)
        return float(self.lib.calculate_peak_frequency(_ptr(src), nt, C.c_float(dt)))

    def propagation(self, vp, rho, shots, dx, dz, dt, nt, pml, fs, freq, filt, precondition, problem,
                    obs=None, pre=None, iteration=1):
        vp, rho = _f32(vp), _f32(rho)
        nx, nz = vp.shape
        n = len(shots)
        obs = [np.zeros((len(s.igx), s.ns), np.float32) if obs is None else _f32(obs[i]).copy()
               for i, s in enumerate(shots)]
        pre = [np.zeros((len(s.igx), s.ns), np.float32) if pre is None else _f32(pre[i]).copy()
               for i, s in enumerate(shots)]
        ro = (Record2D * n)(*[self._record(s, obs[i]) for i, s in enumerate(shots)])
        rp = (Record2D * n)(*[self._record(s, pre[i]) for i, s in enumerate(shots)])
        vpr, rhor = rows(vp), rows(rho)
        grad = np.zeros((nx, nz), np.float32) if problem == 1 else None
        gr = rows(grad) if grad is not None else None
        self.lib.iso_acoustic2d_propagation(vpr, rhor, ro, n, nz, nx, C.c_float(dx), C.c_float(dz),
                                            C.c_float(dt), nt, pml, fs, C.c_float(freq), C.c_float(filt),
                                            precondition, problem, iteration, 0, rp, gr)
        self._keep.clear()
        return pre, grad

    def objective(self, traces, shots):
        tr = [_f32(t) for t in traces]
        recs = (Record2D * len(tr))(*[self._record(s, tr[i]) for i, s in enumerate(shots)])
        v = float(self.lib.calculate_objective_value(recs, len(tr)))
        self._keep.clear()
        return v

    def step_length(self, pre0, pre1, shots):
        a = [_f32(t) for t in pre0]; b = [_f32(t) for t in pre1]
        ra = (Record2D * len(a))(*[self._record(s, a[i]) for i, s in enumerate(shots)])
        rb = (Record2D * len(b))(*[self._record(s, b[i]) for i, s in enumerate(shots)])
        v = float(self.lib.calculate_step_length(ra, rb, len(a)))
        self._keep.clear()
        return v

    def model_perturbation(self, fraction, slow, grad):
        slow, grad = _f32(slow), _f32(grad)
        out = np.zeros_like(grad)
        s = self.lib.compute_model_perturbation(C.c_float(fraction), _ptr(slow), _ptr(grad), _ptr(out), grad.size)
        return float(s), out

    def smooth2d(self, a, N, zdir):
        a = _f32(a)
        out = np.zeros_like(a)
        nx, nz = a.shape
        self.lib.smooth2D(rows(a), rows(out), nx, nz, N, zdir)
        return out
