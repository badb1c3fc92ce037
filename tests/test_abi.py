"""The C-ABI library loads and exports every entry point include/baandi_gpu.h
declares (no GPU needed; no compute call)."""
import ctypes
import os
import re

from baandi_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^int\s+(bg_\w+)\s*\(", text, flags=re.M))
    return names


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_context_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.bg_ctx_create(None, ctypes.byref(h))
    assert rc == _lib.BG_EDEVICE
    assert "device" in _lib.last_error(None)
