"""The C-ABI library: it loads, exports every symbol include/wavefront_gpu.h
declares, and reports argument and device errors as status codes (no aborts),
which is checkable without a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from wavefront_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wavefront_gpu.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    declared = _declared()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(wf_[a-z0-9_]+)$", out, flags=re.M))
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        getattr(lib, s)
    assert sorted(L.EXPORTS) == declared


def test_library_is_built_for_sm100a_only():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", L.LIB_PATH],
                         capture_output=True, text=True).stdout
    archs = set(re.findall(r"sm_\d+a?", out))
    assert archs == {"sm_100a"}, archs


def test_bad_dims_are_an_argument_error_not_a_crash():
    d = L.GridDesc()
    d.nx, d.ny, d.nz = 12, 16, 16
    h = C.c_void_p()
    st = L.lib().wf_create(C.byref(d), C.byref(h))
    assert st == L.WF_ERR_ARG
    assert b"multiples of BLOCK_DIM" in L.lib().wf_last_error(None)


def test_create_without_a_device_reports_status(monkeypatch):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d = L.GridDesc()
    d.nx = d.ny = d.nz = 16
    h = C.c_void_p()
    st = L.lib().wf_create(C.byref(d), C.byref(h))
    assert st == L.WF_ERR_CUDA and not h.value


def test_null_handle_calls_fail_cleanly():
    lib = L.lib()
    assert lib.wf_step(None, 1) == L.WF_ERR_ARG
    assert lib.wf_sync(None) == L.WF_ERR_ARG
    assert lib.wf_destroy(None) == L.WF_OK
    assert lib.wf_status_string(L.WF_ERR_TIMEOUT) == b"device wait timed out"


def _header_arity():
    """Number of parameters of every function the header declares."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(wf_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_signatures_match_the_header():
    """Every binding the Python layer declares has the header's arity (a
    mismatch would pass garbage through the ABI)."""
    lib = L.lib()
    arity = _header_arity()
    checked = 0
    for name in L.EXPORTS:
        fn = getattr(lib, name)
        if fn.argtypes is None:
            continue
        assert len(fn.argtypes) == arity[name], (name, len(fn.argtypes), arity[name])
        checked += 1
    assert checked >= 40


def test_noalloc_argument_errors_before_any_cuda_call():
    """wf_step_fields_noalloc checks its arguments before touching CUDA: null
    pointers, dimensions that are not multiples of 8, grids above its static
    limit, unknown modes and negative step counts are WF_ERR_ARG with a
    message, on a machine with or without a GPU."""
    import numpy as np
    lib = L.lib()
    q = np.zeros((256, 4), np.int32)
    b = (C.c_int32 * 3)(0, 0, 0)
    one = C.c_void_p(16)  # never dereferenced: every case fails before any use

    def call(fields, ids, nx, ny, nz, boundary=b, arith=0, n=1):
        return lib.wf_step_fields_noalloc(fields, ids, L.ptr(q, L.i32p), nx, ny, nz, boundary,
                                          arith, n, None)

    assert call(None, one, 8, 8, 8) == L.WF_ERR_ARG
    assert b"null argument" in lib.wf_noalloc_last_error()
    assert call(one, None, 8, 8, 8) == L.WF_ERR_ARG
    assert call(one, one, 12, 8, 8) == L.WF_ERR_ARG
    assert b"multiples of BLOCK_DIM" in lib.wf_noalloc_last_error()
    assert call(one, one, 72, 64, 64) == L.WF_ERR_ARG
    assert b"exceeds the allocation-free limit of 262144 cells" in lib.wf_noalloc_last_error()
    assert call(one, one, 8, 8, 8, arith=7) == L.WF_ERR_ARG
    assert call(one, one, 8, 8, 8, n=-1) == L.WF_ERR_ARG
    assert call(one, one, 8, 8, 8, boundary=(C.c_int32 * 3)(0, 5, 0)) == L.WF_ERR_ARG
    assert b"unknown boundary kind" in lib.wf_noalloc_last_error()


def test_rust_sys_crate_declares_the_header():
    """The Rust -sys crate (source only: no Rust toolchain here) declares
    every function the header declares, with the header's parameter count."""
    src = open(os.path.join(ROOT, "wavefront_b200", "bindings", "rust", "wavefront-gpu-sys", "src",
                            "lib.rs")).read()
    rust = {}
    for m in re.finditer(r"pub fn (wf_[a-z0-9_]+)\(([^)]*)\)", src):
        params = m.group(2).strip()
        rust[m.group(1)] = 0 if not params else params.count(":")
    assert rust == _header_arity()
