"""The footprint estimate a serving loop admits requests by (fwi_estimate_bytes, host-only)."""
import numpy as np

from fwiedu import engine as E
from fwiedu import models as M
from golden_cases import Case


def survey(nshot, nt, nz=221, nx=601):
    sv = M.line_survey(nz, nx, 12.5, 12.5, 0.001, nt, nshot, M.ricker(nt, 0.001, 10.0, 0.15),
                       spacing_cells=max(1, (nx - 20) // nshot), first_cell=5)
    return M.survey_shots(sv)


def test_estimate_grows_with_the_work():
    c = Case("fs1_small")
    g = E.estimate_bytes(c.shots, c.nz, c.nx, c.nt, c.pml, 1)
    f = E.estimate_bytes(c.shots, c.nz, c.nx, c.nt, c.pml, 0)
    assert g > f > 0
    one = E.estimate_bytes(survey(1, 2001), 221, 601, 2001, 40, 1)
    eight = E.estimate_bytes(survey(8, 2001), 221, 601, 2001, 40, 1)
    longer = E.estimate_bytes(survey(8, 6001), 221, 601, 6001, 40, 1)
    assert one < eight < longer
    # a gradient shot holds its frame block (checkpoint pairs, scratch and kept replay frames),
    # FP64 g and H, three gathers plus samples, and its adjoint source on every step
    Nx, ld, ntr, ns, nt = 681, 304, 601, 4001, 4001
    d = int(round(np.sqrt(2 * 4000)))
    frames = 9 + 2 * ((4000 // d) + 1) + 2 * (d // 5 + 2)
    want = frames * Nx * ld * 4 + 2 * Nx * ld * 8 + 4 * ntr * ns * 4 + nt * ntr * 4 + 2 * 221 * 601 * 4
    per_shot = (E.estimate_bytes(survey(9, 4001), 221, 601, 4001, 40, 1) -
                E.estimate_bytes(survey(1, 4001), 221, 601, 4001, 40, 1)) / 8
    assert want <= per_shot <= 1.1 * want


def test_estimate_rejects_nonsense():
    assert E.estimate_bytes([], 10, 10, 10, 3, 1) == 0
