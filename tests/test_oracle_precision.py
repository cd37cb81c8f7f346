"""FP32 algorithm against its FP64 build: the error every FP32 result carries.

The reference (and therefore the bit-exact CUDA engine) computes in FP32; these
bounds state how far that is from the same algorithm carried in FP64.
"""
import numpy as np

from golden_cases import Case


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_fp32_traces_within_1e5_of_fp64(port32, port64):
    c = Case("fs1_small")
    a, _ = port32.propagation(c.vp, c.rho, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 0.0, 2.0, 1, 0)
    b, _ = port64.propagation(c.vp, c.rho, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 0.0, 2.0, 1, 0)
    for x, y in zip(a, b):
        assert rel(x, y) < 1e-5


def test_fp32_gradient_within_1e3_of_fp64(port32, port64):
    c = Case("fs1_small")
    _, g32 = port32.propagation(c.vp0, c.rho0, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 10.0, 2.0, 1, 1,
                                obs=c.obs)
    _, g64 = port64.propagation(c.vp0, c.rho0, c.shots, c.dx, c.dx, c.dt, c.nt, c.pml, c.fs, 10.0, 2.0, 1, 1,
                                obs=c.obs)
    assert rel(g32, g64) < 1e-3


def test_checkpoint_bookkeeping(port32):
    # d = max(round(sqrt(2(nt-1))), 3) and the pairs (it-1, it) at it % d == 0 (checkpoint.c:47, :66-75)
    for nt, d, n in [(4001, 89, 89), (200, 20, 20), (2, 3, 1), (1, 3, 1), (10, 4, 5)]:
        assert port32.checkpoint_interval(nt) == d
        assert port32.checkpoint_count(nt) == n
