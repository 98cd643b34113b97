"""The C-ABI library loads, exports every symbol include/bn_volume.h
declares, and reports errors instead of crashing -- without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

import barney_b200 as bn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bn_volume.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"BN_API\s+[\w\s\*]+?\b(bnx?\w+)\s*\(", text)))


def test_header_and_wrapper_agree():
    assert declared_symbols() == sorted(bn.EXPORTS)


def test_library_exports_every_declared_symbol():
    path = bn.lib().__dict__.get("_name") or bn.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    # internal symbols stay hidden
    assert not any(s.startswith("_ZN3bnb") for s in exported)


def test_library_loads_and_resolves_symbols():
    L = bn.lib()
    for s in declared_symbols():
        assert getattr(L, s) is not None


def test_errors_are_recorded_not_thrown():
    L = bn.lib()
    L.bnClearLastError()
    L.bnRelease(ctypes.c_void_p(0x1234))
    assert L.bnGetLastError() == 1  # invalid handle
    assert b"handle" in L.bnGetLastErrorString()
    L.bnClearLastError()
    L.bnCommit(None)
    assert L.bnGetLastError() == 1
    L.bnClearLastError()
    with pytest.raises(bn.BarneyError):
        L.bnSet1f(ctypes.c_void_p(8), b"fovy", 1.0)
        bn.check()


def test_context_without_gpu_fails_cleanly():
    L = bn.lib()
    if L.bnPhysicalDeviceCount() > 0:
        pytest.skip("a GPU is present")
    L.bnClearLastError()
    ctx = L.bnContextCreate(1, None, 0, None)
    assert not ctx
    assert L.bnGetLastError() != 0
    L.bnClearLastError()


def test_kernels_compiled_for_sm100a():
    log = open(os.path.join(ROOT, "barney_b200", "csrc", "ptxas.log")).read()
    assert "for 'sm_100a'" in log
    assert "renderKernel" in log
    # the render megakernel must not spill
    blocks = log.split("Function properties for ")
    render = [b for b in blocks[1:] if b.split()[0].startswith("_ZN3bnb12renderKernel")]
    assert render
    for b in render:
        assert "0 bytes spill stores" in b.splitlines()[1]
