"""The PLAIN kernels take cos and sin of each phase from one sincosf call where
the reference calls cosf and sinf separately (MatchedFilter_cuda_kernel.cu:60-63,
SignalTracer_cuda_kernel.cu:442-443, 555-556).  That keeps their results
bit-exact only if the two forms agree for every FP32 input; the probe library's
check compares all 2^32 bit patterns on the device."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_sincosf_matches_separate_calls_for_every_float(cuda):
    from benchkit import probes

    lib = probes.lib()
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    probes.check(lib.geraf_rf_sincos_identity_check(ctypes.c_void_p(count.data_ptr()), stream),
                 "sincos check")
    torch.cuda.synchronize()
    assert int(count.item()) == 0
