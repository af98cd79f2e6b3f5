"""tcgen05 split-BF16 GEMM against an FP64 product (torch matmul on the same device).

Tolerances: hi*hi + hi*lo + lo*hi keeps about 16 significant bits per operand, so the max-norm
error relative to max|C| is bounded by 5e-5 on these random operands; hi*hi alone by 1e-2.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from safire_b200 import capi  # noqa: E402


def _run(M, N, K, batch, ab, bb, nterms, tile_n=0, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(batch if ab else 1, M, K, generator=g, device="cuda", dtype=torch.float64)
    B = torch.randn(batch if bb else 1, N, K, generator=g, device="cuda", dtype=torch.float64)
    C = torch.full((batch, M, N), float("nan"), device="cuda", dtype=torch.float32)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(capi.lib().sfq_gemm_split_bf16(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, batch, int(ab),
                                              int(bb), nterms, tile_n, st))
    ref = torch.matmul(A, B.transpose(1, 2)).expand(batch, M, N)
    torch.cuda.synchronize()
    err = (C.double() - ref).abs().max().item() / ref.abs().max().item()
    return err


@pytest.mark.parametrize("shape", [
    (256, 256, 256, 1, 0, 0, 0),
    (200, 100, 136, 1, 0, 0, 0),     # ragged M, N, K tails (TMA zero fill)
    (300, 520, 2400, 1, 0, 0, 256),
    (100, 800, 800, 3, 1, 1, 128),   # batched, one row tile per batch
    (130, 64, 512, 2, 0, 1, 64),     # shared A
    (512, 1000, 2400, 1, 0, 0, 128),
])
def test_split_bf16_gemm_three_terms(shape):
    M, N, K, batch, ab, bb, tn = shape
    assert _run(M, N, K, batch, ab, bb, 3, tn) < 5e-5


def test_split_bf16_gemm_one_term():
    assert _run(256, 384, 512, 1, 0, 0, 1) < 1e-2


def test_split_bf16_gemm_rejects_bad_k():
    rc = capi.lib().sfq_gemm_split_bf16(ctypes.c_void_p(256), ctypes.c_void_p(256), ctypes.c_void_p(256), 8, 8, 12,
                                        1, 0, 0, 3, 0, None)
    assert rc == 1
