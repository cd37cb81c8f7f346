"""fwi_smooth2d_noalloc, the smoothing entry point for callers that cannot allocate
device memory (serving loops with a fixed device budget, host code between captured
graph segments): its output must equal the existing smooth2D entry point applied as
the FWI loop applies it (z pass, then x pass) and the oracle's smoothing, on calls in a
row through the one shared scratch array -- a larger grid, then a smaller one, a grid
narrower than the window, and a call in place -- and oversized grids must be refused.

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


def noalloc(a, rz, rx, in_place=False):
    import torch
    L = E.lib()
    nx, nz = a.shape
    din = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    dout = din if in_place else torch.full_like(din, float("nan"))
    rc = L.fwi_smooth2d_noalloc(C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr()), nx, nz, rz, rx, None)
    torch.cuda.synchronize()
    assert rc == E.FWI_OK, rc
    return dout.cpu().numpy()


def test_noalloc_smoothing_matches_smooth2d_on_consecutive_calls(port32):
    c = Case("fs1_small")
    rng = np.random.default_rng(3)
    calls = [
        ((3.0 * c.vp0 + c.grad).astype(np.float32), 3, 2, False),  # the larger grid first
        (c.grad, 1, 1, False),                                       # then a smaller one
        (rng.standard_normal((5, 7)).astype(np.float32), 32, 32, False),  # window wider than both axes
        (c.grad, 2, 3, True),                                        # in place
    ]
    outs = [noalloc(a, rz, rx, ip) for a, rz, rx, ip in calls]
    for (a, rz, rx, _), got in zip(calls, outs):
        want = smooth2d_twice(a, rz, rx)
        assert np.array_equal(got, want), f"max diff {np.abs(got - want).max()}"
        oracle = port32.smooth2d(port32.smooth2d(a, rz, 1), rx, 0)
        assert np.array_equal(got, oracle), f"oracle: max diff {np.abs(got - oracle).max()}"
    # the FWI loop's smoothing of the golden gradient (acoustic2d_fwi.c:418-419, rz = rx = 1)
    assert np.array_equal(outs[1], c["grad_smooth"])


def test_noalloc_smoothing_rejects_oversized_grids():
    import torch
    L = E.lib()
    d = torch.zeros(16, device="cuda")
    p = C.c_void_p(d.data_ptr())
    assert L.fwi_smooth2d_noalloc(p, p, 4096, 2048, 1, 1, None) == E.FWI_ERR_ARG
    assert L.fwi_smooth2d_noalloc(p, p, 4, 4, 0, 1, None) == E.FWI_ERR_ARG
    assert L.fwi_smooth2d_noalloc(p, p, 4, 4, 1, 33, None) == E.FWI_ERR_ARG
