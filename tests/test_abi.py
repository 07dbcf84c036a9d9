"""The C-ABI library loads and exports every symbol include/grico_b200.h declares."""
import ctypes
import os
import re

import grico_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "grico_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|double|const char\*)\s+(grico_\w+)\s*\(", text, flags=re.M)))


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
    import numpy as np

    desc = L.GricoPlanDesc()
    desc.dim = 3
    desc.form = L.GRICO_FORM_MASS_DIFFUSION
    offsets = np.zeros(1, dtype=np.int64)
    desc.red_offsets = L.ptr(offsets, ctypes.c_int64)
    handle = ctypes.c_void_p()
    rc = L.lib().grico_plan_create(ctypes.byref(desc), ctypes.byref(handle))
    assert rc == L.GRICO_ERR_NO_DEVICE
    assert b"no CUDA device" in L.lib().grico_last_error()


def test_descriptor_validation_runs_before_cuda():
    """A malformed descriptor is rejected on the host with a precise message."""
    import numpy as np

    desc = L.GricoPlanDesc()
    desc.dim = 3
    desc.form = 99
    handle = ctypes.c_void_p()
    assert L.lib().grico_plan_create(ctypes.byref(desc), ctypes.byref(handle)) == L.GRICO_ERR_UNSUPPORTED_FORM
    desc.form = L.GRICO_FORM_MASS_DIFFUSION
    desc.n_full = 4
    offsets = np.zeros(5, dtype=np.int64)
    desc.red_offsets = L.ptr(offsets, ctypes.c_int64)
    batch = (L.GricoCellBatchDesc * 1)()
    batch[0].n_cells = 1
    batch[0].degree[:] = [1, 1, 1]
    batch[0].qpoints[:] = [2, 2, 2]
    bad = np.full(8, 7, dtype=np.int32)  # dof 7 >= n_full
    h = np.ones(3)
    batch[0].map_index = L.ptr(bad, ctypes.c_int32)
    batch[0].cell_size = L.ptr(h, ctypes.c_double)
    desc.n_batches = 1
    desc.batches = batch
    assert L.lib().grico_plan_create(ctypes.byref(desc), ctypes.byref(handle)) == L.GRICO_ERR_INVALID
    assert b"out of range" in L.lib().grico_last_error()


def test_conv_tc_weight_bytes():
    """Packed tensor-core weights: 27 taps x Ci/8 chunks x N rows x 16 bytes, N = Co rounded up to
    a multiple of 32; shapes the kernel does not serve report -1 (host-only, no device needed)."""
    lib = L.lib()
    assert lib.grico_conv_tc_weight_bytes(32, 32) == 27 * 4 * 32 * 16
    assert lib.grico_conv_tc_weight_bytes(32, 1) == 27 * 4 * 32 * 16
    assert lib.grico_conv_tc_weight_bytes(16, 40) == 27 * 2 * 64 * 16
    assert lib.grico_conv_tc_weight_bytes(2, 32) == -1
    assert lib.grico_conv_tc_weight_bytes(64, 128) == -1  # shared memory over 227 KB
