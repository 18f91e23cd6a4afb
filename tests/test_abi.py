"""CPU-side checks of the C-ABI library: it loads without a GPU and exports every entry point
that include/moist2d.h declares (no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SO = os.path.join(ROOT, "moist2d_b200", "libmoist2d_sm100a.so")


def declared_functions():
    src = open(os.path.join(ROOT, "include", "moist2d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(moist_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def built():
    if not os.path.exists(SO):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "moist2d_b200", "csrc")], check=True)
    return SO


def test_library_exports_every_declared_symbol(built):
    L = C.CDLL(built)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", built], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (moist_\w+)", out))
    assert set(names) <= exported


def test_abi_version_and_status_strings(built):
    L = C.CDLL(built)
    assert L.moist_abi_version() == 1
    L.moist_status_string.restype = C.c_char_p
    assert L.moist_status_string(0) == b"ok"
    assert L.moist_status_string(1) == b"NaN detected"


def test_binding_lists_every_export():
    from moist2d_b200 import _lib
    assert set(_lib.EXPORTS) == set(declared_functions())


def test_ctx_create_rejects_bad_params_without_gpu(built):
    """Argument validation happens before any CUDA call."""
    import numpy as np
    from moist2d_b200.params import Params
    L = C.CDLL(built)
    p = Params(np.float32, Nx=4, Nz=4, H=430.0, dz0=100.0, z_fact=1.05)
    cp = p.to_c()
    cp.nz = 1  # a one-level column has no w-p system
    ctx = C.c_void_p()
    assert L.moist_ctx_create(C.byref(cp), 0, 0, C.byref(ctx)) == 2  # MOIST_ERR_ARG
