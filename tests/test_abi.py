"""The C-ABI library: it loads, exports every entry point include/fwi_b200.h declares,
and its host-only functions behave (no device needed).  On a machine without a GPU
the engine refuses to start instead of falling back to the CPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from fwiedu import engine as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fwi_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^FWI_API[^(]*?\b([A-Za-z_][A-Za-z_0-9]*)\(", txt, re.M)))


def test_header_declares_the_reference_entry_points():
    names = declared()
    for ref_name in ("iso_acoustic2d_propagation", "iso_acoustic2d_propagation_engine",
                     "alloc_acoustic2dCheckPoint", "free_acoustic2dCheckPoint", "calculate_memory_cost_checkpoint",
                     "calculate_objective_value", "calculate_step_length", "compute_model_perturbation",
                     "compute_adjoint_source2d", "smooth2D", "apply_gradient_precondition",
                     "apply_gradient_shot_precondition"):
        assert ref_name in names


def test_library_exports_every_declared_symbol():
    path = E.build()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in declared() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    lib = C.CDLL(path)
    for n in declared():
        assert hasattr(lib, n)


def test_version_and_memory_cost():
    L = E.lib()
    assert b"sm_100a" in L.fwi_version()
    # calculate_memory_cost_checkpoint: (nCheckPoint + d - 2) frames of NX*NZ floats, in GB
    nt, NX, NZ = 4001, 681, 301
    d, n = 89, 89
    want = np.float32((n + d - 2) * NZ * NX * 4) / np.float32(1024.0 ** 3)
    assert L.calculate_memory_cost_checkpoint(nt, NX, NZ) == pytest.approx(float(want), rel=1e-6)
    assert L.fwi_checkpoint_interval(4001) == 89


def test_no_cpu_fallback_without_device():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = E.lib().fwi_ctx_create(C.byref(h), 0, C.c_size_t(0))
    assert rc == E.FWI_ERR_NODEVICE
    with pytest.raises(E.FwiError):
        E.Context(0)
