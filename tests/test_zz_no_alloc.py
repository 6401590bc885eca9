"""fe_mass_weight_noalloc: the mass reduction for callers that cannot allocate
device memory (their own pool owns the GPU memory, or their loop must not
enter cudaMalloc/cudaFree). It keeps its partial sums in a fixed array inside
the library; the caller passes the populations and the 2-double output in its
own device memory. Checked here against the engine's own entry point
(fe_current_mass) on two calls in a row, the second on a later state, so a
stale counter or partial left by the first call would show. Collected last
(file name) so a failure does not hide the other GPU tests."""
import ctypes as C

import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import MultiPhaseGPU, _capi

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the FP64 parity tolerance of the other tests


def test_noalloc_mass_matches_engine_on_two_calls(require_gpu):
    import torch
    case = make_case("grf_mrt_mass")
    e = MultiPhaseGPU(case.params, case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        e.record_target_mass()
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        out = torch.zeros(2, dtype=torch.float64, device="cuda")
        for call in range(2):
            if call == 1:
                e.run(10)
            h, _ = e.download_state()
            m_engine = e.current_mass()
            hd = torch.from_numpy(h).to("cuda")
            torch.cuda.synchronize()
            _capi.check(_capi.lib.fe_mass_weight_noalloc(C.c_void_p(hd.data_ptr()), e.n,
                                                         C.c_void_p(out.data_ptr()), stream))
            torch.cuda.synchronize()
            m, w = out.cpu().numpy()
            c = h.reshape(19, -1).sum(0)
            w_ref = float(np.maximum(c * (1.0 - c), 0.0).sum())
            assert abs(m - m_engine) <= TOL * abs(m_engine), (call, m, m_engine)
            assert abs(w - w_ref) <= TOL * abs(w_ref), (call, w, w_ref)
    finally:
        e.free()


def test_noalloc_rejects_sizes_beyond_scratch(require_gpu):
    import torch
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = _capi.lib.fe_mass_weight_noalloc(C.c_void_p(out.data_ptr()), 33554432 + 1, C.c_void_p(out.data_ptr()),
                                          None)
    assert rc == _capi.FE_ERR_ARG
    assert b"exceeds the fixed scratch capacity" in _capi.lib.fe_last_error()


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 3 * 2048 + 5])
def test_noalloc_block_edges(require_gpu, n):
    """Sizes around the 2048-site block split (one partial block, exactly one
    block, one site over, several blocks and a ragged tail): M and W against
    a numpy sum on two calls in a row, so a stale counter would show."""
    import torch
    gen = torch.Generator(device="cuda").manual_seed(n)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        h = torch.rand(19 * n, dtype=torch.float64, device="cuda", generator=gen) * (2.0 / 19.0)
        torch.cuda.synchronize()
        _capi.check(_capi.lib.fe_mass_weight_noalloc(C.c_void_p(h.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                                     stream))
        torch.cuda.synchronize()
        m, w = out.cpu().numpy()
        c = h.cpu().numpy().reshape(19, n).sum(0)
        m_ref = float(c.sum())
        w_ref = float(np.maximum(c * (1.0 - c), 0.0).sum())
        assert abs(m - m_ref) <= TOL * abs(m_ref), (n, call, m, m_ref)
        assert abs(w - w_ref) <= TOL * max(abs(w_ref), 1e-300), (n, call, w, w_ref)
