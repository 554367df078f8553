"""liblsmgpu.so loads without a GPU and exports every symbol that
include/lsmgpu/lsmgpu.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from lsmlib_b200 import abi, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lsmgpu", "lsmgpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", src)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"if", "defined", "sizeof"}
    return sorted({n for n in names if n not in skip and
                   (n.startswith("lsm3d") or n.startswith("lsmgpu_") or
                    n.startswith("compute") or n.startswith("solve"))})


def test_header_declares_all_reference_symbols():
    decl = set(declared_functions())
    missing = [s for s in abi.SIGNATURES if s not in decl]
    assert not missing, missing


def test_library_exports_every_declared_symbol():
    lib = gpu.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_exports_reference_symbols_without_prefix():
    lib = ctypes.CDLL(gpu.LIB_PATH)
    for sym in abi.SIGNATURES:
        assert hasattr(lib, sym), sym


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(FileNotFoundError):
        gpu.load.__wrapped__(str(tmp_path / "nope.so")) if hasattr(gpu.load, "__wrapped__") \
            else _load_fresh(str(tmp_path / "nope.so"))


def _load_fresh(path):
    saved = gpu._lib
    gpu._lib = None
    try:
        return gpu.load(path)
    finally:
        gpu._lib = saved


def test_workspace_calls_reject_a_null_workspace():
    """The workspace setters check their handle on the host before any CUDA
    call, so a null workspace is an error code, not a crash."""
    lib = gpu.load()
    null = ctypes.c_void_p()
    err_null = 2   # LSMGPU_ERR_NULL_POINTER
    assert lib.lsmgpu_workspace_set_fp64_policy(null, 8) == err_null
    assert lib.lsmgpu_workspace_set_fp64_band(null, 16.0, 1) == err_null
    assert lib.lsmgpu_workspace_set_host_async(null, 1) == err_null
    assert lib.lsmgpu_workspace_sync(null) == err_null
