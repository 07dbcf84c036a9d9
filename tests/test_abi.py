"""The C-ABI library loads and exports every symbol include/grico_b200.h declares."""
import ctypes
import os
import re

import grico_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "grico_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|double|const char\*)\s+(grico_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)


def test_plan_create_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        return
    desc = L.GricoPlanDesc()
    desc.dim = 3
    desc.form = L.GRICO_FORM_MASS_DIFFUSION
    handle = ctypes.c_void_p()
    rc = L.lib().grico_plan_create(ctypes.byref(desc), ctypes.byref(handle))
    assert rc == L.GRICO_ERR_NO_DEVICE
    assert b"no CUDA device" in L.lib().grico_last_error()
