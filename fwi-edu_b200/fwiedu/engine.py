"""ctypes binding of libfwi_b200.so (the B200 engine) -- the host-side mirror of the
reference's propagation interface.

Two ways in, as in the C-ABI (include/fwi_b200.h):

* ``propagation(...)`` calls the drop-in ``fwi_iso_acoustic2d_propagation`` with
  Record2D shot records and host arrays, exactly as acoustic2d_modeling.c and
  acoustic2d_fwi.c call ``iso_acoustic2d_propagation`` (propagation.h:133-142);
* ``Context`` wraps the native device-resident API (fwi_ctx_*).

There is no CPU fallback: loading fails loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libfwi_b200.so")
CSRC = os.path.join(PKG, "csrc")

FWI_OK, FWI_ERR_ARG, FWI_ERR_CUDA, FWI_ERR_NOMEM, FWI_ERR_UNSUPPORTED, FWI_ERR_NODEVICE, FWI_ERR_STATE = range(7)
PATH_PLAIN, PATH_BATCHED = 0, 1

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_fpp = C.POINTER(_fp)


class FwiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"status {code}: {msg}")
        self.code = code


class Record2D(C.Structure):
    """Shot record, layout of observation.h:18-48."""
    _fields_ = [("shotID", C.c_int), ("sx", C.c_float), ("sz", C.c_float), ("isx", C.c_int),
                ("isz", C.c_int), ("fpeak", C.c_float), ("src", _fp), ("gx", _fp), ("gz", _fp),
                ("igx", _ip), ("igz", _ip), ("sampleRate", C.c_int), ("ntr", C.c_int),
                ("ns", C.c_int), ("dtr", C.c_float), ("dt", C.c_float), ("ix_min", C.c_int),
                ("ix_max", C.c_int), ("traces_vx", _fpp), ("traces_vz", _fpp), ("traces_p", _fpp),
                ("precond", _fpp), ("grad", _fpp)]


class FwiShot(C.Structure):
    _fields_ = [("shotID", C.c_int), ("isx", C.c_int), ("isz", C.c_int), ("ntr", C.c_int),
                ("ns", C.c_int), ("sampleRate", C.c_int), ("ix_min", C.c_int), ("ix_max", C.c_int),
                ("dt", C.c_float), ("dtr", C.c_float), ("fpeak", C.c_float),
                ("src", _fp), ("igx", _ip), ("igz", _ip)]


class FwiStats(C.Structure):
    _fields_ = [("ms", C.c_double), ("cell_updates", C.c_double), ("kernel_launches", C.c_longlong),
                ("graph_launches", C.c_longlong), ("device_bytes", C.c_size_t)]


class IterParams(C.Structure):
    """fwi_iter_params: one iteration of the FWI loop (acoustic2d_fwi.c:411-465)."""
    _fields_ = [("rx", C.c_int), ("rz", C.c_int), ("precondition", C.c_int), ("filter", C.c_int),
                ("freq", C.c_float), ("waterdepth", C.c_int), ("vp_water", C.c_float), ("rho_water", C.c_float),
                ("vpmin", C.c_float), ("vpmax", C.c_float), ("rhomin", C.c_float), ("rhomax", C.c_float),
                ("gardner", C.c_int), ("path", C.c_int)]


class IterResult(C.Structure):
    _fields_ = [("fun1", C.c_float), ("fun2", C.c_float), ("steplen", C.c_float), ("scalar", C.c_float),
                ("ms", C.c_double), ("cell_updates", C.c_double), ("kernel_launches", C.c_longlong)]


_lib = None
_lock = threading.Lock()


def build(force: bool = False) -> str:
    """Compile the library in-tree (nvcc, sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", CSRC, "-j4"], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = C.CDLL(LIB_PATH)
            L.fwi_last_error.restype = C.c_char_p
            L.fwi_version.restype = C.c_char_p
            L.fwi_ctx_traces_device.restype = C.c_void_p
            L.fwi_ctx_gradient_device.restype = C.c_void_p
            L.calculate_memory_cost_checkpoint.restype = C.c_float
            L.fwi_request_bytes.restype = C.c_size_t
            L.fwi_estimate_bytes.restype = C.c_size_t
            _lib = L
    return _lib


def _check(rc):
    if rc != FWI_OK:
        raise FwiError(rc, lib().fwi_last_error().decode(errors="replace"))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a, t=_fp):
    return a.ctypes.data_as(t)


def rows(a: np.ndarray):
    """float** view (alloc2float layout) of a C-contiguous (n2, n1) float32 array."""
    assert a.dtype == np.float32 and a.flags.c_contiguous
    n2 = a.shape[0]
    n1 = int(np.prod(a.shape[1:])) if a.ndim > 1 else 1
    arr = (_fp * max(n2, 1))()
    base = a.ctypes.data
    for i in range(n2):
        arr[i] = C.cast(base + i * n1 * 4, _fp)
    return arr


class _Keep(list):
    pass


def make_records(shots, traces, keep):
    """Record2D array for the Shot list with the given per-shot (ntr, ns) trace buffers."""
    recs = (Record2D * len(shots))()
    for i, s in enumerate(shots):
        igx, igz, src = _i32(s.igx), _i32(s.igz), _f32(s.src)
        gx = ((igx + s.ix_min).astype(np.float32) * np.float32(s.dtr)).astype(np.float32)
        gz = igz.astype(np.float32)
        rp = rows(traces[i])
        keep += [igx, igz, src, gx, gz, rp, traces[i]]
        r = recs[i]
        r.shotID = s.shotID; r.sx = s.sx; r.sz = s.sz; r.isx = s.isx; r.isz = s.isz; r.fpeak = s.fpeak
        r.src = _ptr(src); r.gx = _ptr(gx); r.gz = _ptr(gz); r.igx = _ptr(igx, _ip); r.igz = _ptr(igz, _ip)
        r.sampleRate = s.sampleRate; r.ntr = len(igx); r.ns = s.ns; r.dtr = s.dtr; r.dt = s.dt
        r.ix_min = s.ix_min; r.ix_max = s.ix_max
        r.traces_p = C.cast(rp, _fpp)
    return recs


def propagation(vp, rho, shots, dx, dz, dt, nt, pml, fs, freq, filt, precondition, problem,
                obs=None, pre=None, iteration=1, path: str | None = None):
    """Drop-in call: iso_acoustic2d_propagation semantics, host arrays in and out.
    Returns (pre gathers, grad or None)."""
    L = lib()
    if path is not None:
        os.environ["FWI_PATH"] = path
    vp, rho = _f32(vp), _f32(rho)
    nx, nz = vp.shape
    keep = _Keep()
    obs = [np.zeros((len(s.igx), s.ns), np.float32) if obs is None else _f32(obs[i]).copy()
           for i, s in enumerate(shots)]
    pre = [np.zeros((len(s.igx), s.ns), np.float32) if pre is None else _f32(pre[i]).copy()
           for i, s in enumerate(shots)]
    ro = make_records(shots, obs, keep)
    rp = make_records(shots, pre, keep)
    vpr, rhor = rows(vp), rows(rho)
    grad = np.zeros((nx, nz), np.float32) if problem == 1 else None
    gr = rows(grad) if grad is not None else None
    rc = L.fwi_iso_acoustic2d_propagation(vpr, rhor, ro, len(shots), nz, nx, C.c_float(dx), C.c_float(dz),
                                          C.c_float(dt), nt, pml, fs, C.c_float(freq), C.c_float(filt),
                                          precondition, problem, iteration, 0, rp, gr)
    _check(rc)
    return pre, grad


class Executor:
    """Continuous batching (fwi_exec_*): runs of several contexts advanced by the same step
    launches; a run added while others are in flight joins at the next launch."""

    def __init__(self, device: int = 0):
        self.L = lib()
        self.h = C.c_void_p()
        _check(self.L.fwi_exec_create(C.byref(self.h), device))

    def add(self, ctx, problem, freq=0.0, filt=2, precondition=1):
        _check(self.L.fwi_exec_add(self.h, ctx.h, int(problem), C.c_float(freq), int(filt), int(precondition)))

    def step(self, launches=0):
        """Issue up to `launches` step launches (0: until the batch is empty); runs left."""
        a = C.c_int()
        _check(self.L.fwi_exec_step(self.h, int(launches), C.byref(a)))
        return a.value

    def poll(self, ctx):
        d, st = C.c_int(), C.c_int()
        _check(self.L.fwi_exec_poll(self.h, ctx.h, C.byref(d), C.byref(st)))
        return bool(d.value), st.value

    def launches(self):
        n = C.c_longlong()
        _check(self.L.fwi_exec_launches(self.h, C.byref(n)))
        return n.value

    def close(self):
        if self.h:
            self.L.fwi_exec_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# fwi_allreduce_fn: int (*)(double *dev, size_t count, void *stream, void *user)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p)


class Context:
    """Device-resident engine context (fwi_ctx_*)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        self.L = lib()
        self.h = C.c_void_p()
        _check(self.L.fwi_ctx_create(C.byref(self.h), device, C.c_size_t(budget_bytes)))
        self._keep = []
        self.shots = []

    def close(self):
        if self.h:
            self.L.fwi_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_model(self, vp, rho, dx, dz, dt, nt, pml, fs):
        vp, rho = _f32(vp), _f32(rho)
        nx, nz = vp.shape
        self.nx, self.nz = nx, nz
        _check(self.L.fwi_ctx_set_model(self.h, _ptr(vp), _ptr(rho), nz, nx, C.c_float(dx), C.c_float(dz),
                                        C.c_float(dt), nt, pml, fs))

    def set_model_device(self, vp_ptr, rho_ptr, nz, nx, dx, dz, dt, nt, pml, fs):
        self.nx, self.nz = nx, nz
        _check(self.L.fwi_ctx_set_model_device(self.h, C.c_void_p(vp_ptr), C.c_void_p(rho_ptr), nz, nx,
                                               C.c_float(dx), C.c_float(dz), C.c_float(dt), nt, pml, fs))

    def set_shots(self, shots):
        arr = (FwiShot * len(shots))()
        keep = []
        for i, s in enumerate(shots):
            igx, igz, src = _i32(s.igx), _i32(s.igz), _f32(s.src)
            keep += [igx, igz, src]
            a = arr[i]
            a.shotID = s.shotID; a.isx = s.isx; a.isz = s.isz; a.ntr = len(igx); a.ns = s.ns
            a.sampleRate = s.sampleRate; a.ix_min = s.ix_min; a.ix_max = s.ix_max
            a.dt = s.dt; a.dtr = s.dtr; a.fpeak = s.fpeak
            a.src = _ptr(src); a.igx = _ptr(igx, _ip); a.igz = _ptr(igz, _ip)
        _check(self.L.fwi_ctx_set_shots(self.h, arr, len(shots)))
        self.shots = list(shots)

    def set_observed(self, obs):
        obs = [_f32(o) for o in obs]
        p = (_fp * len(obs))(*[_ptr(o) for o in obs])
        _check(self.L.fwi_ctx_set_observed(self.h, p))

    def run(self, problem, freq=0.0, filt=2, precondition=1, path=PATH_BATCHED):
        _check(self.L.fwi_ctx_run(self.h, problem, C.c_float(freq), filt, precondition, path))

    def traces(self, i):
        s = self.shots[i]
        out = np.empty((len(s.igx), s.ns), np.float32)
        _check(self.L.fwi_ctx_get_traces(self.h, i, _ptr(out)))
        return out

    def gradient(self):
        out = np.empty((self.nx, self.nz), np.float32)
        _check(self.L.fwi_ctx_get_gradient(self.h, _ptr(out)))
        return out

    def objective(self):
        v = C.c_double()
        _check(self.L.fwi_ctx_objective(self.h, C.byref(v)))
        return v.value

    def fwi_iteration(self, params: IterParams):
        r = IterResult()
        _check(self.L.fwi_ctx_fwi_iteration(self.h, C.byref(params), C.byref(r)))
        return {k: getattr(r, k) for k, _ in IterResult._fields_}

    def model(self):
        vp = np.empty((self.nx, self.nz), np.float32)
        rho = np.empty_like(vp)
        _check(self.L.fwi_ctx_get_model(self.h, _ptr(vp), _ptr(rho)))
        return vp, rho

    def pass_stats(self):
        """Device time and step launches of the last run's forward and adjoint passes."""
        fm, am = C.c_double(), C.c_double()
        fl, al = C.c_longlong(), C.c_longlong()
        _check(self.L.fwi_ctx_pass_stats(self.h, C.byref(fm), C.byref(fl), C.byref(am), C.byref(al)))
        return {"fwd_ms": fm.value, "fwd_launches": fl.value, "adj_ms": am.value, "adj_launches": al.value}

    def set_verbose(self, verbose, iteration=1, shot_interval=0, snap_interval=0, directory=None):
        """The reference's intermediate files (fwi_ctx_set_verbose): verbose 1 per-shot traces and
        gradients and the stacked gradient of a gradient run, verbose 2 also wavefield snapshots.
        Intervals <= 0 come from the shotInterval / snapInterval environment variables."""
        d = None if directory is None else str(directory).encode()
        _check(self.L.fwi_ctx_set_verbose(self.h, int(verbose), int(iteration), int(shot_interval),
                                          int(snap_interval), d))

    def set_allreduce(self, fn):
        """Install the exchange hook of a shot-sharded run (fwi_ctx_set_allreduce).

        ``fn(dev_ptr, count, stream_ptr)`` must replace ``count`` FP64 values at device address
        ``dev_ptr`` by their sum over all ranks, ordered on the engine's CUDA stream
        ``stream_ptr`` (see fwiedu.dist.device_hook).  ``None`` removes the hook."""
        if fn is None:
            self._ar = None
            _check(self.L.fwi_ctx_set_allreduce(self.h, None, None))
            return

        def _cb(dev, count, stream, user):
            try:
                fn(int(dev or 0), int(count), int(stream or 0))
                return 0
            except Exception:  # reported to the engine as a failed exchange
                import traceback
                traceback.print_exc()
                return 1

        self._ar = ALLREDUCE_FN(_cb)  # keep the thunk alive as long as the context
        _check(self.L.fwi_ctx_set_allreduce(self.h, self._ar, None))

    def launch_shape(self):
        """Shape of the last step launch (fwi_ctx_launch_shape, fwi_ctx_launch_variant), and whether
        the last pass ran as one persistent wavefront launch (fwi_ctx_launch_persistent)."""
        v = [C.c_int() for _ in range(6)]
        _check(self.L.fwi_ctx_launch_shape(self.h, C.byref(v[0]), C.byref(v[1]), C.byref(v[2])))
        _check(self.L.fwi_ctx_launch_variant(self.h, C.byref(v[3]), C.byref(v[4])))
        _check(self.L.fwi_ctx_launch_persistent(self.h, C.byref(v[5])))
        keys = ("tile_columns", "ring_depth", "shots_per_block", "groups_per_thread", "blocks_per_sm", "persistent")
        return {k: x.value for k, x in zip(keys, v)}

    def stats(self):
        s = FwiStats()
        _check(self.L.fwi_ctx_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in FwiStats._fields_}


# ---------------------------------------------------------------- serving (fwi_server_*)
REQ_MODEL, REQ_GRADIENT = 0, 1
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(4)


class FwiRequest(C.Structure):
    _fields_ = [("kind", C.c_int), ("nz", C.c_int), ("nx", C.c_int), ("dx", C.c_float), ("dz", C.c_float),
                ("dt", C.c_float), ("nt", C.c_int), ("pml", C.c_int), ("fs", C.c_int), ("vp", _fp), ("rho", _fp),
                ("shots", C.POINTER(FwiShot)), ("nshot", C.c_int), ("obs", _fpp), ("freq", C.c_float),
                ("filter", C.c_int), ("precondition", C.c_int), ("traces", _fpp), ("grad", _fp)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("bytes", C.c_size_t), ("queue_ms", C.c_double),
                ("run_ms", C.c_double), ("total_ms", C.c_double), ("objective", C.c_double),
                ("cell_updates", C.c_double), ("error", C.c_char * 256)]


class ServerReport(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("rejected", C.c_longlong), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("p50_queue_ms", C.c_double), ("p99_queue_ms", C.c_double), ("wall_s", C.c_double),
                ("cell_updates", C.c_double), ("shots_modeled", C.c_double), ("shot_gradients", C.c_double),
                ("budget", C.c_size_t), ("peak_bytes", C.c_size_t), ("max_active", C.c_int),
                ("peak_active", C.c_int)]


def _shot_array(shots, keep):
    arr = (FwiShot * len(shots))()
    for i, s in enumerate(shots):
        igx, igz, src = _i32(s.igx), _i32(s.igz), _f32(s.src)
        keep += [igx, igz, src]
        a = arr[i]
        a.shotID = s.shotID; a.isx = s.isx; a.isz = s.isz; a.ntr = len(igx); a.ns = s.ns
        a.sampleRate = s.sampleRate; a.ix_min = s.ix_min; a.ix_max = s.ix_max
        a.dt = s.dt; a.dtr = s.dtr; a.fpeak = s.fpeak
        a.src = _ptr(src); a.igx = _ptr(igx, _ip); a.igz = _ptr(igz, _ip)
    keep.append(arr)
    return arr


def request(kind, vp, rho, dx, dz, dt, nt, pml, fs, shots, obs=None, freq=10.0, filt=2, precondition=1):
    """A fwi_request with its input and output buffers (kept in the returned holder):
    returns (FwiRequest, holder) where holder["traces"] / holder["grad"] receive the results."""
    keep = []
    vp, rho = _f32(vp), _f32(rho)
    nx, nz = vp.shape
    keep += [vp, rho]
    r = FwiRequest()
    r.kind = kind; r.nz = nz; r.nx = nx; r.dx = dx; r.dz = dz; r.dt = dt; r.nt = nt; r.pml = pml; r.fs = fs
    r.vp = _ptr(vp); r.rho = _ptr(rho)
    r.shots = C.cast(_shot_array(shots, keep), C.POINTER(FwiShot)); r.nshot = len(shots)
    if obs is not None:
        obs = [_f32(o) for o in obs]
        keep += obs
        po = (_fp * len(obs))(*[_ptr(o) for o in obs])
        keep.append(po)
        r.obs = C.cast(po, _fpp)
    r.freq = freq; r.filter = filt; r.precondition = precondition
    traces = [np.zeros((len(s.igx), s.ns), np.float32) for s in shots]
    pt = (_fp * len(traces))(*[_ptr(t) for t in traces])
    keep += [traces, pt]
    r.traces = C.cast(pt, _fpp)
    grad = np.zeros((nx, nz), np.float32) if kind == REQ_GRADIENT else None
    if grad is not None:
        r.grad = _ptr(grad)
    keep.append(r)
    return r, {"traces": traces, "grad": grad, "keep": keep}


class Server:
    """The serving loop (fwi_server_*): concurrent, footprint-admitted requests on one GPU."""

    def __init__(self, device=0, budget_bytes=0, max_active=4):
        self.L = lib()
        self.h = C.c_void_p()
        _check(self.L.fwi_server_create(C.byref(self.h), device, C.c_size_t(budget_bytes), max_active))
        self.pending = {}

    def bytes(self, req):
        return int(self.L.fwi_request_bytes(C.byref(req)))

    def submit(self, req, holder):
        rid = C.c_longlong()
        _check(self.L.fwi_server_submit(self.h, C.byref(req), C.byref(rid)))
        self.pending[rid.value] = holder
        return rid.value

    def wait(self, rid, timeout_s=-1.0):
        info = RequestInfo()
        rc = self.L.fwi_server_wait(self.h, C.c_longlong(rid), C.c_double(timeout_s), C.byref(info))
        out = {k: getattr(info, k) for k, _ in RequestInfo._fields_}
        out["error"] = info.error.decode(errors="replace")
        if rc == FWI_OK:
            holder = self.pending.pop(rid)
            out["traces"], out["grad"] = holder["traces"], holder["grad"]
        return out

    def report(self):
        s = ServerReport()
        _check(self.L.fwi_server_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerReport._fields_}

    def close(self):
        if self.h:
            self.L.fwi_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_bytes(shots, nz, nx, nt, pml, problem, filt=2):
    """fwi_estimate_bytes: device bytes one context needs for the run (host-side, no GPU)."""
    L = lib()
    keep = []
    arr = _shot_array(shots, keep)
    return int(L.fwi_estimate_bytes(arr, len(shots), nz, nx, nt, pml, problem, filt))
