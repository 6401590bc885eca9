"""Batch and server entry points without a GPU: argument checks return a
status, and creation reports the missing device instead of crashing."""
import ctypes as C

import pytest

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
    # the in-place population layout: FP64 / FP32 storage only; known layouts only
    bad = _capi.FeServerConfig(0, 0, 0.1, 10, _capi.STORAGE["f16g"], 0, 1)
    assert lib.fe_server_create(C.byref(bad), C.byref(h)) == _capi.FE_ERR_ARG
    bad = _capi.FeServerConfig(0, 0, 0.1, 10, _capi.FE_F32, 0, 2)
    assert lib.fe_server_create(C.byref(bad), C.byref(h)) == _capi.FE_ERR_ARG
    assert lib.fe_server_submit(None, None) == _capi.FE_ERR_ARG
    assert lib.fe_server_destroy(None) == 0
    assert lib.fe_server_free_result(None) == 0
    if not torch.cuda.is_available():
        ok = _capi.FeServerConfig(0, 0, 0.1, 10, _capi.FE_F32, 0)
        assert lib.fe_server_create(C.byref(ok), C.byref(h)) == _capi.FE_ERR_NO_DEVICE
        ok = _capi.FeServerConfig(0, 0, 0.1, 10, _capi.FE_F32, 0, 1)
        assert lib.fe_server_create(C.byref(ok), C.byref(h)) == _capi.FE_ERR_NO_DEVICE


def test_struct_sizes_match_header(tmp_path):
    """The ctypes mirrors have the C structs' sizes (a mismatch would corrupt
    requests): the header compiled by the host C compiler tells."""
    import os
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    names = {"fe_request": _capi.FeRequest, "fe_result": _capi.FeResult, "fe_server_stats": _capi.FeServerStats,
             "fe_server_config": _capi.FeServerConfig, "fe_params": _capi.FeParams,
             "fe_tracer_config": _capi.FeTracerConfig, "fe_tune_report": _capi.FeTuneReport,
             "fe_fields": _capi.FeFields, "fe_open_bnd": _capi.FeOpenBnd}
    src = tmp_path / "sizes.c"
    src.write_text("#include <stdio.h>\n#include \"felbm_b200.h\"\nint main(void){\n" +
                   "".join('printf("%%zu\\n", sizeof(%s));\n' % n for n in names) + "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    for (n, cls), size in zip(names.items(), got):
        assert C.sizeof(cls) == size, n
