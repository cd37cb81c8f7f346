"""The 2-D wavenumber filters as drop-in entry points (lowpass2d / bandpass2d, common.c:1042-1284).

Pinned twice: against the reference's own output on a smoothed random field
(tests/golden/aux_wavenumber.npz, made by tests/golden/make_golden.py from the reference's C
sources with FFTW) -- the in-place taper of the input bit for bit, the filtered field within
rel-L2 1e-5 -- and against numpy's FFT run the way the reference runs FFTW (taper, edge-replicated
pad, rfft2, the reference's float window on the stored half plane, irfft2, / (Nz Nx), crop) on
other shapes, spacings and band edges.  The GPU computes the DFTs of the padded field's own sizes
as Bluestein transforms (hand-written FFT kernels, FP64 where a block holds the transform).
"""
import ctypes as C
import os

import numpy as np
import pytest

from fwiedu import engine as E

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
F32 = np.float32


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def run(fn, s, dz, dx, kpass, kcut, out=None):
    """fn on s ([nx][nz], modified in place as the reference modifies it); returns the output."""
    nx, nz = s.shape
    y = np.zeros_like(s) if out is None else out
    fn(E.rows(s), nz, nx, C.c_float(dz), C.c_float(dx), C.c_float(kpass), C.c_float(kcut), E.rows(y))
    return y


def taper_coefs(n):
    x = F32(np.pi) * np.arange(n + 1, dtype=F32) / F32(n)
    return (F32(0.5) * (F32(1.0) + np.cos(x, dtype=F32))).astype(F32)


def np_taper(s, lt, lr):
    """taper_traces (common.c:796-895) with nz as the time axis and nx as the trace axis."""
    nx, nz = s.shape
    lt, lr = min(lt, nz // 3), min(lr, nx // 3)
    if lt > 0:
        t = taper_coefs(lt)
        s[:, : lt + 1] *= t[::-1]
        s[:, nz - lt - 1:] *= t
    if lr > 0:
        r = taper_coefs(lr)
        s[: lr + 1, :] *= r[::-1, None]
        s[nx - lr - 1:, :] *= r[:, None]


def angular(n, d):
    """generate_frequency (common.c:333-361) in float."""
    df = F32(2.0) * F32(np.pi) / F32(n * F32(d))
    f = np.zeros(n, F32)
    nf = n // 2 + 1
    for it in range(1, nf):
        f[it] = F32(it) * df
        if n - it >= nf:
            f[n - it] = -f[it]
    return f


def np_window(filt, Nx, Nz, dx, dz, kpass, kcut):
    """The reference's window on the stored half plane [Nx][Nz/2+1], float expressions."""
    two_pi = F32(2.0) * F32(np.pi)
    KX = (angular(Nx, dx) / two_pi)[:, None]
    KZ = (angular(Nz, dz) / two_pi)[None, : Nz // 2 + 1]
    k = np.sqrt(KX * KX + KZ * KZ, dtype=F32)
    kp, kc, pi = F32(kpass), F32(kcut), F32(np.pi)
    band = (k >= kp) & (k <= kc)
    if filt == 0:
        w = np.where(k < kp, F32(1.0), F32(0.0)).astype(F32)
        w[band] = F32(0.5) * (F32(1.0) + np.cos(pi * (k[band] - kp) / (kc - kp), dtype=F32))
    else:
        w = np.zeros_like(k)
        lo = k < kp
        w[lo] = F32(0.5) * (F32(1.0) + np.cos(pi * (kp - k[lo]) / kp, dtype=F32))
        w[band] = F32(0.5) * (F32(1.0) + np.cos(pi * (k[band] - kp) / (kc - kp), dtype=F32))
    return w


def np_filter(field, filt, dz, dx, kpass, kcut):
    s = field.astype(F32).copy()
    nx, nz = s.shape
    lx = int(np.floor(F32(4) / (F32(kpass) * F32(dx)) + F32(0.5)))
    lz = int(np.floor(F32(4) / (F32(kpass) * F32(dz)) + F32(0.5)))
    np_taper(s, lz, lx)
    pad = 10 * max(lx, lz)
    sp = np.pad(s.astype(np.float64), pad, mode="edge")
    Nx, Nz = sp.shape
    spec = np.fft.rfft2(sp) * np_window(filt, Nx, Nz, dx, dz, kpass, kcut)
    y = np.fft.irfft2(spec, s=(Nx, Nz))
    return s, y[pad: pad + nx, pad: pad + nz]


@pytest.mark.parametrize("kind", ["low", "band"])
def test_wavenumber_filter_matches_reference_output(kind):
    g = np.load(os.path.join(HERE, "golden", "aux_wavenumber.npz"))
    L = E.lib()
    fn = L.lowpass2d if kind == "low" else L.bandpass2d
    s = np.ascontiguousarray(g["field"], F32)
    y = run(fn, s, float(g["dz"]), float(g["dx"]), float(g[kind + "_kpass"]), float(g[kind + "_kcut"]))
    assert np.array_equal(s, g[kind + "_tapered_input"])  # the reference tapers its input in place
    assert rel(y, g[kind + "_out"]) <= 1e-5


@pytest.mark.parametrize("filt,nx,nz,dz,dx,kpass,kcut", [
    (0, 70, 40, 12.5, 10.0, 0.02, 0.04),
    (1, 33, 57, 10.0, 10.0, 0.03, 0.06),
    (0, 128, 64, 5.0, 8.0, 0.05, 0.08),
    (1, 201, 96, 10.0, 12.5, 0.012, 0.03),
])
def test_wavenumber_filter_matches_fft(filt, nx, nz, dz, dx, kpass, kcut):
    L = E.lib()
    fn = L.lowpass2d if filt == 0 else L.bandpass2d
    rng = np.random.default_rng(nx * nz + filt)
    field = (2000.0 + 300.0 * rng.standard_normal((nx, nz))).astype(F32)
    tap, want = np_filter(field, filt, dz, dx, kpass, kcut)
    s = field.copy()
    y = run(fn, s, dz, dx, kpass, kcut)
    assert np.abs(s - tap).max() <= 1e-6 * np.abs(tap).max()  # numpy's cos may differ from cosf by an ulp
    assert rel(y, want) <= 1e-5


def test_wavenumber_filter_in_place_and_bad_band():
    L = E.lib()
    rng = np.random.default_rng(7)
    field = rng.standard_normal((50, 30)).astype(F32)
    a = field.copy()
    y = run(L.lowpass2d, a, 10.0, 10.0, 0.03, 0.05)
    b = field.copy()
    run(L.lowpass2d, b, 10.0, 10.0, 0.03, 0.05, out=b)  # s_filter == s, as the reference allows
    assert np.array_equal(b, y)
    c = field.copy()
    out = np.full_like(c, 3.0)
    run(L.bandpass2d, c, 10.0, 10.0, 0.05, 0.05, out=out)  # kcut <= kpass: error, nothing changed
    assert np.array_equal(c, field) and (out == 3.0).all()
