"""fwi_smooth2d_noalloc, the smoothing entry point for callers that cannot allocate
device memory (serving loops with a fixed device budget, host code between captured
graph segments): its output must equal the existing smooth2D entry point applied as
the FWI loop applies it (z pass, then x pass), on two calls in a row through the one
shared scratch array, and oversized grids must be refused.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from fwiedu import engine as E
from golden_cases import Case

pytestmark = pytest.mark.gpu


def smooth2d_twice(a, rz, rx):
    L = E.lib()
    nx, nz = a.shape
    a = np.ascontiguousarray(a, np.float32)
    t = np.zeros_like(a)
    o = np.zeros_like(a)
    L.smooth2D(E.rows(a), E.rows(t), nx, nz, rz, 1)
    L.smooth2D(E.rows(t), E.rows(o), nx, nz, rx, 0)
    return o


def test_noalloc_smoothing_matches_smooth2d_on_consecutive_calls():
    import torch
    L = E.lib()
    c = Case("fs1_small")
    calls = [(c.grad, 1, 1), ((3.0 * c.vp0 + c.grad).astype(np.float32), 3, 2)]
    outs = []
    for a, rz, rx in calls:
        nx, nz = a.shape
        din = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
        dout = torch.full_like(din, float("nan"))
        rc = L.fwi_smooth2d_noalloc(C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr()), nx, nz, rz, rx, None)
        torch.cuda.synchronize()
        assert rc == E.FWI_OK
        outs.append(dout.cpu().numpy())
    for (a, rz, rx), got in zip(calls, outs):
        want = smooth2d_twice(a, rz, rx)
        assert np.array_equal(got, want), f"max diff {np.abs(got - want).max()}"


def test_noalloc_smoothing_rejects_oversized_grids():
    import torch
    L = E.lib()
    d = torch.zeros(16, device="cuda")
    p = C.c_void_p(d.data_ptr())
    assert L.fwi_smooth2d_noalloc(p, p, 4096, 2048, 1, 1, None) == E.FWI_ERR_ARG
    assert L.fwi_smooth2d_noalloc(p, p, 4, 4, 0, 1, None) == E.FWI_ERR_ARG
    assert L.fwi_smooth2d_noalloc(p, p, 4, 4, 1, 33, None) == E.FWI_ERR_ARG
