"""The C ABI library builds for sm_100a, loads, and exports every symbol include/*.h declares.

No compute call is made here (this file runs without a GPU).
"""
import ctypes
import os
import subprocess

import pytest

from untangling26_b200 import _native, build


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    assert lib is not None


def test_every_declared_symbol_is_exported():
    path = build.build()
    names = _native.declared_symbols()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    lib = _native.load(path)
    for n in names:
        assert hasattr(lib, n)


def test_binding_signatures_cover_header():
    names = set(_native.declared_symbols())
    bound = set(_native._SIGS)
    assert names == bound, f"header/binding mismatch: {sorted(names ^ bound)}"


def test_sm100a_code_in_library():
    path = build.build()
    out = subprocess.run(["cuobjdump", "--list-elf", path], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_ctx_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = _native.load()
    h = ctypes.c_void_p()
    st = lib.u26_ctx_create(0, None, ctypes.byref(h))
    assert st == 6  # U26_ERR_NO_DEVICE
