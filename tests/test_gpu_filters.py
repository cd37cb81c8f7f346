"""The residual filters and the trace interpolation as drop-in entry points
(apply_traces_lowpass / apply_traces_bandpass / interpolate_traces, common.c:482-794, and
compute_adjoint_source2d with filters 0/1, optimization.c:300-419), against numpy's FFT run
the way the reference runs FFTW: r2c, the reference's float window on the non-negative
frequencies, c2r, / n (the interpolation: zero-stuffing, complex FFT, rectangular window of
height r, inverse, real part / n).  FP32 GEMMs with the equivalent operators: rel-L2 <= 1e-5.
"""
import ctypes as C

import numpy as np
import pytest

from fwiedu import engine as E
from golden_cases import Case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def window(filt, n, fpass, fcut, dt):
    """The reference's window (float expressions, PI double in the bandpass argument)."""
    f32 = np.float32
    df = f32(1.0) / f32(n * f32(dt))
    w = np.zeros(n, np.float32)
    for it in range(n):
        f = f32(it) * df
        if filt == 0:
            if f < fpass:
                w[it] = 1.0
            elif f <= fcut:
                w[it] = f32(0.5) * (f32(1.0) + np.cos(f32(np.pi) * (f - f32(fpass)) / (f32(fcut) - f32(fpass)),
                                                       dtype=np.float32))
        else:
            if f < fpass:
                w[it] = f32(0.5) * (f32(1.0) + f32(np.cos(np.float64(np.pi) * (f32(fpass) - f) / f32(fpass))))
            elif f <= fcut:
                w[it] = f32(0.5) * (f32(1.0) + f32(np.cos(np.float64(np.pi) * (f - f32(fpass)) /
                                                          (f32(fcut) - f32(fpass)))))
    return w


def np_filter(x, filt, fpass, fcut, dt):
    n = x.shape[-1]
    w = window(filt, n, fpass, fcut, dt)[: n // 2 + 1]
    return np.fft.irfft(np.fft.rfft(x.astype(np.float64), axis=-1) * w, n=n, axis=-1)


def rows(a):
    return E.rows(a)


@pytest.mark.parametrize("filt,n", [(0, 301), (1, 301), (0, 4001), (1, 512)])
def test_traces_filters(filt, n):
    L = E.lib()
    rng = np.random.default_rng(n + filt)
    ntr, dt = 23, 0.002
    x = rng.standard_normal((ntr, n)).astype(np.float32)
    y = np.zeros_like(x)
    fn = L.apply_traces_lowpass if filt == 0 else L.apply_traces_bandpass
    fn(rows(x), rows(y), n, ntr, C.c_float(12.0), C.c_float(24.0), C.c_float(dt))
    assert rel(y, np_filter(x, filt, 12.0, 24.0, dt)) <= 1e-5
    fn(rows(x), rows(x), n, ntr, C.c_float(12.0), C.c_float(24.0), C.c_float(dt))  # in place, as the reference allows
    assert np.array_equal(x, y)


@pytest.mark.parametrize("r,nt", [(2, 151), (3, 100), (4, 1001)])
def test_interpolate_traces(r, nt):
    L = E.lib()
    rng = np.random.default_rng(r * nt)
    ntr = 9
    x = rng.standard_normal((ntr, nt)).astype(np.float32)
    ns = (nt - 1) * r + 1
    y = np.zeros((ntr, ns), np.float32)
    L.interpolate_traces(rows(x), ntr, nt, r, rows(y))
    z = np.zeros((ntr, ns), np.complex128)
    z[:, ::r] = x
    spec = np.fft.fft(z, axis=-1)
    nkeep = ns // (2 * r)
    w = np.zeros(ns)
    w[:nkeep] = r
    w[ns - nkeep + 1:] = r
    want = np.fft.ifft(spec * w, axis=-1).real
    assert rel(y, want) <= 1e-5


@pytest.mark.parametrize("name", ["filt0", "filt1"])
def test_adjoint_source_entry_point_filters(name):
    """compute_adjoint_source2d with filters 0/1 on the engine's own predicted traces."""
    c = Case(name)
    pre, _ = E.propagation(c.vp0, c.rho0, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 0.0, 2.0, c.precondition, 0)
    L = E.lib()
    vpr = rows(np.ascontiguousarray(c.vp0, np.float32))
    for i, s in enumerate(c.shots):
        keep = []
        p_ = [np.ascontiguousarray(pre[i])]
        o_ = [np.ascontiguousarray(c.obs[i], np.float32)]
        a_ = [np.zeros_like(pre[i])]
        rp = E.make_records([s], p_, keep)
        ro = E.make_records([s], o_, keep)
        ra = E.make_records([s], a_, keep)
        L.compute_adjoint_source2d(rp, ro, vpr, C.c_float(10.0), int(c.filter), ra)
        assert rel(a_[0], c.adj[i]) <= 1e-5, f"shot {i}: {rel(a_[0], c.adj[i]):.2e}"
