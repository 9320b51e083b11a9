"""The C-ABI library loads without a GPU and exports every entry point that
include/hrrt_gpu.h declares (no compute calls here)."""
import ctypes
import os
import re

import hrrt_reconstruction_b200 as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "hrrt_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(hrrt_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "hrrt_ctx_create" in names and "hrrt_osem" in names and "hrrt_fp_pair" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(H.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_library_is_built_for_sm100a_only():
    """The build recipe targets sm_100a and nothing else."""
    from hrrt_reconstruction_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_context_without_gpu_fails_cleanly():
    """No GPU here: creation reports a CUDA error instead of aborting."""
    import torch
    if torch.cuda.is_available():
        return
    g = H.hrrt_geometry(span=9)
    try:
        H.Context(g)
    except H.HrrtError as e:
        assert "cuda" in str(e).lower() or "device" in str(e).lower()
    else:
        raise AssertionError("context creation should fail without a GPU")
