"""Batch and server entry points without a GPU: argument checks return a
status, and creation reports the missing device instead of crashing."""
import ctypes as C

import torch

from felbm_gpu_b200 import _capi


def test_batch_arguments():
    lib = _capi.lib
    assert lib.fe_batch_destroy(None) == 0
    assert lib.fe_batch_run(None, 1) == _capi.FE_ERR_ARG
    assert lib.fe_batch_add(None, None) == _capi.FE_ERR_ARG
    assert lib.fe_batch_create(0, None) == _capi.FE_ERR_ARG
    if not torch.cuda.is_available():
        h = C.c_void_p()
        assert lib.fe_batch_create(0, C.byref(h)) == _capi.FE_ERR_NO_DEVICE
        assert not h.value


def test_server_arguments():
    lib = _capi.lib
    h = C.c_void_p()
    bad = _capi.FeServerConfig(0, 0, 0.1, 0, _capi.FE_F32, 0)  # chunk_steps 0
    assert lib.fe_server_create(C.byref(bad), C.byref(h)) == _capi.FE_ERR_ARG
    bad = _capi.FeServerConfig(0, 0, 1.5, 10, _capi.FE_F32, 0)
    assert lib.fe_server_create(C.byref(bad), C.byref(h)) == _capi.FE_ERR_ARG
    bad = _capi.FeServerConfig(0, 0, 0.1, 10, 9, 0)
    assert lib.fe_server_create(C.byref(bad), C.byref(h)) == _capi.FE_ERR_ARG
    assert lib.fe_server_submit(None, None) == _capi.FE_ERR_ARG
    assert lib.fe_server_destroy(None) == 0
    assert lib.fe_server_free_result(None) == 0
    if not torch.cuda.is_available():
        ok = _capi.FeServerConfig(0, 0, 0.1, 10, _capi.FE_F32, 0)
        assert lib.fe_server_create(C.byref(ok), C.byref(h)) == _capi.FE_ERR_NO_DEVICE


def test_struct_sizes_match_header():
    # sizes of the C structs (gcc, x86-64): a mismatch would corrupt requests
    assert C.sizeof(_capi.FeRequest) == 456
    assert C.sizeof(_capi.FeResult) == 328
    assert C.sizeof(_capi.FeServerStats) == 112
    assert C.sizeof(_capi.FeServerConfig) == 32
