"""Loading of the reference's golden vectors (tests/golden/*.npz) into shot lists."""
from __future__ import annotations

import glob
import os

import numpy as np

from fwiedu.models import Shot

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The propagation cases (aux_*.npz hold fixtures of single functions, demo_*.npz the expected
    outputs of whole front-end runs)."""
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("aux_", "demo_")))


class Case:
    def __init__(self, name):
        self.name = name
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.z = z
        for k in ("nz", "nx", "nt", "pml", "fs", "precondition", "nshot"):
            setattr(self, k, int(z[k]))
        self.dt = float(z["dt"])
        self.dx = float(z["dx"])
        self.vp, self.rho = z["vp"], z["rho"]
        sc, sf, src = z["shot_scalars"], z["shot_floats"], z["src"]
        self.shots = []
        for i in range(self.nshot):
            shotID, isx, isz, ns, sr, ixmin, ixmax = (int(v) for v in sc[i])
            dt, dtr, fpeak, sx, sz = (float(v) for v in sf[i])
            self.shots.append(Shot(shotID=shotID, isx=isx, isz=isz, igx=z[f"igx{i}"], igz=z[f"igz{i}"], ns=ns,
                                   sampleRate=sr, ix_min=ixmin, ix_max=ixmax, dt=dt, dtr=dtr, fpeak=fpeak, src=src,
                                   sx=sx, sz=sz))
        self.obs = [z[f"obs{i}"] for i in range(self.nshot)]
        # residual filter of the gradient case (optimization.c:368-415) and whether an FFT stage
        # (filters 0/1, or interpolation for sampleRate > 1) lies between the forward traces and
        # the adjoint source: those results are compared within a tolerance, the rest bit for bit
        self.filter = float(z["filter"]) if "filter" in z else 2.0
        self.fft = int(self.filter) in (0, 1) or any(s.sampleRate > 1 for s in self.shots)
        self.has_grad = "grad" in z
        if self.has_grad:
            self.vp0, self.rho0 = z["vp0"], z["rho0"]
            self.adj = [z[f"adj{i}"] for i in range(self.nshot)]
            self.grad = z["grad"]
            self.vp1, self.rho1 = z["vp1"], z["rho1"]
            self.has_res = "res0" in z
            if self.has_res:
                self.res = [z[f"res{i}"] for i in range(self.nshot)]

    def __getitem__(self, k):
        return self.z[k]
