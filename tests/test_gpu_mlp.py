"""Tensor-core (tcgen05) kernels of the learned surrogate against CPU
arithmetic on the same bf16 operands."""
import ctypes

import numpy as np
import pytest

from eu3d_b200 import gpu

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("M,N,K", [(128, 16, 16), (128, 128, 64), (256, 48, 80), (384, 256, 128), (128, 64, 144)])
@pytest.mark.parametrize("accumulate", [0, 1])
def test_gemm_tc_matches_cpu(M, N, K, accumulate):
    torch = _torch()
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    C0 = torch.randn(M, N, generator=g, dtype=torch.float32)
    ref = A.double() @ B.double().T + (C0.double() if accumulate else 0.0)
    dA, dB, dC = A.cuda(), B.cuda(), C0.cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    L = gpu.load_library()
    rc = L.eu3d_gemm_bf16(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, N, K, accumulate, err.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.eu3d_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = dC.cpu().double()
    scale = ref.abs().max().item()
    assert (got - ref).abs().max().item() <= 1e-5 * scale * max(1, K / 16)


def test_gemm_tc_rejects_bad_shapes():
    torch = _torch()
    L = gpu.load_library()
    buf = torch.zeros(256 * 256, dtype=torch.bfloat16, device="cuda")
    out = torch.zeros(256 * 256, dtype=torch.float32, device="cuda")
    p, o = buf.data_ptr(), out.data_ptr()
    assert L.eu3d_gemm_bf16(p, p, o, 100, 16, 16, 0, None, None) == -1
    assert L.eu3d_gemm_bf16(p, p, o, 128, 24, 16, 0, None, None) == -1
    assert L.eu3d_gemm_bf16(p, p, o, 128, 16, 8, 0, None, None) == -1
    assert L.eu3d_gemm_bf16(p + 2, p, o, 128, 16, 16, 0, None, None) == -1
