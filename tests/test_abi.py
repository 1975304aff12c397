"""The C ABI: libspmx.so loads on a machine without a GPU, exports every entry
point include/spmx.h declares, and the Python binding covers them all."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    hdr = open(os.path.join(ROOT, "include", "spmx.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(spmx_[a-z0-9_]+)\s*\(", hdr)))


def test_library_loads_and_exports_header():
    import spmx
    out = subprocess.run(["nm", "-D", "--defined-only", spmx.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(spmx_\w+)", out))
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_declares_every_header_symbol():
    import spmx
    assert set(header_symbols()) == set(spmx.declared_symbols())


def test_no_torch_types_in_header():
    hdr = open(os.path.join(ROOT, "include", "spmx.h")).read()
    assert "torch" not in hdr.lower().replace("no torch", "")
    assert 'extern "C"' in hdr


def test_create_without_gpu_reports_no_device():
    import ctypes
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from spmx import abi
    h = ctypes.c_void_p()
    rc = abi.lib.spmx_create(10, 10, 5, ctypes.byref(h))
    assert rc == abi.ERR_NO_DEVICE
    assert "no CUDA device" in abi.last_error()


def test_invalid_arguments_rejected_on_host():
    import ctypes
    from spmx import abi
    assert abi.lib.spmx_create(-1, 3, 3, ctypes.byref(ctypes.c_void_p())) == abi.ERR_INVALID_VALUE
    assert abi.lib.spmx_destroy(None) == abi.SUCCESS
    assert abi.lib.spmx_set_stream(None, None) == abi.ERR_INVALID_VALUE
    k = ctypes.c_int()
    assert abi.lib.spmx_select(None, ctypes.byref(k)) == abi.ERR_INVALID_VALUE


def test_kernels_built_for_sm100a():
    """The library carries sm_100a device code (checked from the build line,
    not by reading the binary)."""
    mk = open(os.path.join(ROOT, "spmspv-adaptive_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk
