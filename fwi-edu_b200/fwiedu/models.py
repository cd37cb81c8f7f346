"""Seeded synthetic models, wavelets and acquisitions for the FWI-EDU workloads.

No dataset ships with the workloads this package is measured on, so every model is
generated from a seed:

* ``layered_model`` -- water (1500 m/s) in the top rows, then layers whose interface
  depths are drawn from the seed with dips within +-10 degrees, layer velocities evenly
  spaced between ``vmin`` and ``vmax``, plus Gaussian anomalies of +-``anom_dv`` m/s.
* ``gardner`` -- rho = 310 vp^0.25 (kg/m^3), water density elsewhere fixed.
* ``ricker`` -- a Ricker wavelet of peak frequency ``f`` delayed by ``t0``.
* ``smooth_model`` -- 2-D Gaussian smoothing with the water layer kept fixed (the
  starting model of a gradient workload).

Arrays follow the reference's column-major layout: shape ``(nx, nz)`` in C order, so the
flat index is ``ix*nz + iz`` with z fastest (``alloc2float(nz, nx)``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def ricker(nt: int, dt: float, f: float = 10.0, t0: float = 0.15) -> np.ndarray:
    t = np.arange(nt, dtype=np.float64) * dt - t0
    a = (math.pi * f * t) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


def layered_model(nz: int, nx: int, seed: int, n_layers: int = 8, water_rows: int = 20,
                  vmin: float = 1600.0, vmax: float = 4500.0, vwater: float = 1500.0,
                  n_anom: int = 3, anom_dv: float = 300.0, anom_sigma: float = 10.0,
                  max_dip_deg: float = 10.0) -> np.ndarray:
    """Layered velocity model (m/s), shape (nx, nz), float32."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx, dtype=np.float64)
    z = np.arange(nz, dtype=np.float64)
    vel = np.linspace(vmin, vmax, n_layers)
    # interface k (k = 1..n_layers-1) separates layer k-1 and k; the first layer starts below the water
    depths = np.sort(rng.uniform(water_rows + 2, nz - 4, size=n_layers - 1))
    dips = np.tan(np.deg2rad(rng.uniform(-max_dip_deg, max_dip_deg, size=n_layers - 1)))
    xc = 0.5 * (nx - 1)
    vp = np.empty((nx, nz), dtype=np.float64)
    layer = np.zeros((nx, nz), dtype=np.int64)
    for k in range(n_layers - 1):
        zi = depths[k] + dips[k] * (x - xc)  # interface depth per column, in cells (dx == dz)
        layer += (z[None, :] >= zi[:, None]).astype(np.int64)
    layer = np.clip(layer, 0, n_layers - 1)
    vp[:] = vel[layer]
    for _ in range(n_anom):
        ax = rng.uniform(0.1 * nx, 0.9 * nx)
        az = rng.uniform(water_rows + anom_sigma, nz - anom_sigma)
        amp = anom_dv * (1.0 if rng.uniform() < 0.5 else -1.0)
        vp += amp * np.exp(-(((x[:, None] - ax) ** 2 + (z[None, :] - az) ** 2) / (2.0 * anom_sigma**2)))
    vp[:, :water_rows] = vwater
    return vp.astype(np.float32)


def gardner(vp: np.ndarray, water_rows: int = 20, rho_water: float = 1000.0) -> np.ndarray:
    rho = (310.0 * np.power(vp.astype(np.float64), 0.25)).astype(np.float32)
    rho[:, :water_rows] = rho_water
    return rho


def smooth_model(vp: np.ndarray, sigma: float, water_rows: int = 20) -> np.ndarray:
    """Separable Gaussian smoothing (edge-replicated), water rows kept."""
    r = int(math.ceil(3.0 * sigma))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    a = vp.astype(np.float64)
    for axis in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[axis] = (r, r)
        ap = np.pad(a, pad, mode="edge")
        out = np.zeros_like(a)
        for i, w in enumerate(k):
            sl = [slice(None), slice(None)]
            sl[axis] = slice(i, i + a.shape[axis])
            out += w * ap[tuple(sl)]
        a = out
    a[:, :water_rows] = vp[:, :water_rows]
    return a.astype(np.float32)


@dataclass
class Survey:
    """A 2-D acquisition in grid indices (global x, global z), as create_grid_observe2d builds it."""
    nz: int
    nx: int
    dx: float
    dz: float
    dt: float
    nt: int
    src: np.ndarray                      # (nt,) float32 wavelet
    sx: list = field(default_factory=list)   # source grid x per shot (global)
    sz: list = field(default_factory=list)   # source grid z per shot
    gx: list = field(default_factory=list)   # receiver grid x per shot (global), int32 arrays
    gz: list = field(default_factory=list)   # receiver grid z per shot, int32 arrays
    sample_rate: int = 1
    rule: str = ""

    @property
    def nshot(self) -> int:
        return len(self.sx)


def line_survey(nz: int, nx: int, dx: float, dz: float, dt: float, nt: int, nshot: int,
                src: np.ndarray, spacing_cells: float | None = None, first_cell: int = 0,
                sdepth_cells: int = 1, gdepth_cells: int = 1, sample_rate: int = 1) -> Survey:
    """Shots on a line, one receiver per column at ``gdepth_cells``.

    When ``nshot`` shots at ``spacing_cells`` do not fit in the model, the spacing is
    reduced to fit: shot k sits at round(first + k * (nx - 1 - first) / (nshot - 1)).
    The rule used is recorded in ``Survey.rule``.
    """
    sv = Survey(nz, nx, dx, dz, dt, nt, np.asarray(src, np.float32), sample_rate=sample_rate)
    if spacing_cells is None or first_cell + spacing_cells * (nshot - 1) > nx - 1:
        span = (nx - 1 - first_cell)
        pos = [int(round(first_cell + k * span / max(nshot - 1, 1))) for k in range(nshot)]
        sv.rule = f"reduced spacing: ix_k = round({first_cell} + k*{span}/{max(nshot - 1, 1)})"
    else:
        pos = [int(round(first_cell + k * spacing_cells)) for k in range(nshot)]
        sv.rule = f"spacing {spacing_cells} cells from {first_cell}"
    g = np.arange(nx, dtype=np.int32)
    for p in pos:
        sv.sx.append(p)
        sv.sz.append(sdepth_cells)
        sv.gx.append(g.copy())
        sv.gz.append(np.full(nx, gdepth_cells, dtype=np.int32))
    return sv


def window(gx: np.ndarray, nx: int, pad: int = 30) -> tuple[int, int]:
    """Per-shot model window: receivers +-30 cells, clipped (observation.c:397-405)."""
    return max(int(gx.min()) - pad, 0), min(int(gx.max()) + pad, nx - 1)


def peak_frequency(src: np.ndarray, nt: int, dt: float) -> float:
    """fpeak = df * argmax |rfft(src)| with df = 1/(nt dt) in float (common.c:363-413)."""
    amp = np.abs(np.fft.rfft(np.asarray(src[:nt], np.float64)))
    i = int(np.argmax(amp))
    df = np.float32(1.0) / (np.float32(nt) * np.float32(dt))
    return float(np.float32(np.float32(i) * df))


@dataclass
class Shot:
    """One shot record in the engine's terms (the fields of Record2D the engine reads).

    ``isx``/``igx`` are window-local x indices, ``isz``/``igz`` global z indices, all
    without the absorbing layer, exactly as create_grid_observe2d leaves them.
    """
    shotID: int
    isx: int
    isz: int
    igx: np.ndarray
    igz: np.ndarray
    ns: int
    sampleRate: int
    ix_min: int
    ix_max: int
    dt: float
    dtr: float
    fpeak: float
    src: np.ndarray
    sx: float = 0.0
    sz: float = 0.0

    @property
    def ntr(self) -> int:
        return int(len(self.igx))

    @property
    def nxx(self) -> int:
        return self.ix_max - self.ix_min + 1


def receiver_interval(gx_m: np.ndarray) -> float:
    """Mean receiver spacing accumulated in float as init_observe2d does (observation.c:316-321)."""
    gx = np.asarray(gx_m, np.float32)
    acc = np.float32(0.0)
    for i in range(len(gx) - 1, 0, -1):
        acc = np.float32(acc + np.float32(gx[i] - gx[i - 1]))
    return float(np.float32(acc / np.float32(len(gx) - 1))) if len(gx) > 1 else 0.0


def survey_shots(sv: Survey, window_pad: int = 30) -> list:
    """Shot records of a Survey, with the per-shot model window of create_grid_observe2d."""
    ns = (sv.nt - 1) // sv.sample_rate + 1
    fpk = peak_frequency(sv.src, sv.nt, sv.dt)
    shots = []
    for k in range(sv.nshot):
        gx = np.asarray(sv.gx[k], np.int32)
        lo, hi = window(gx, sv.nx, window_pad)
        shots.append(Shot(shotID=k + 1, isx=int(sv.sx[k]) - lo, isz=int(sv.sz[k]),
                          igx=(gx - lo).astype(np.int32), igz=np.asarray(sv.gz[k], np.int32),
                          ns=ns, sampleRate=sv.sample_rate, ix_min=lo, ix_max=hi,
                          dt=float(np.float32(np.float32(sv.dt) * sv.sample_rate)),
                          dtr=receiver_interval(gx.astype(np.float32) * np.float32(sv.dx)),
                          fpeak=fpk, src=sv.src, sx=float(sv.sx[k] * sv.dx), sz=float(sv.sz[k] * sv.dz)))
    return shots
