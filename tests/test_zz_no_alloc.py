"""The allocation-free mixed density matrix against the workspace entry point.

sfq_mixed_density_matrix_noalloc exists for callers that cannot allocate device memory (a host
program whose allocator owns all of it, an FFI binding without a CUDA runtime, a loop that must
not pay for cudaMalloc).  It keeps its scratch in a fixed array inside the library, shared by
every call, so this test makes two calls in a row with different inputs -- the second one runs
on whatever the first left in the array -- and compares both to sfq_mixed_density_matrix with
a caller workspace, at the 1e-10 relative tolerance the other parity tests use.  This file is
collected last so a failure here does not hide the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from safire_b200 import afqmc, capi  # noqa: E402

REL = 1e-10


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _inputs(seed, W, M, N, complex_trial):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(N, M)) + (1j * rng.normal(size=(N, M)) if complex_trial else 0)
    B = rng.normal(size=(W, M, N)) + 1j * rng.normal(size=(W, M, N))
    A = torch.as_tensor(np.ascontiguousarray(A)).cuda()
    return A, torch.as_tensor(B).cuda()


def _noalloc(A, B):
    W, M, N = B.shape
    C = torch.full((W, N, M), complex(7.0, -3.0), dtype=torch.complex128, device="cuda")
    ov = torch.zeros(W, dtype=torch.complex128, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(capi.lib().sfq_mixed_density_matrix_noalloc(A.data_ptr(), int(A.dtype == torch.complex128),
                                                           B.data_ptr(), C.data_ptr(), ov.data_ptr(), W, M, N, stream))
    torch.cuda.synchronize()
    return C.cpu().numpy(), ov.cpu().numpy()


def test_noalloc_matches_workspace_entry_point_twice():
    for seed, (W, M, N, cplx) in enumerate([(37, 96, 24, False), (64, 128, 32, True)]):
        A, B = _inputs(seed, W, M, N, cplx)
        C_ref, ov_ref = afqmc.MixedDensityMatrix(A, B, compact=True)
        torch.cuda.synchronize()
        C, ov = _noalloc(A, B)
        assert _rel(C, C_ref.cpu().numpy()) < REL
        assert _rel(ov, ov_ref.cpu().numpy()) < REL


def test_noalloc_rejects_oversize_request():
    cap = capi.lib().sfq_noalloc_scratch_bytes()
    assert cap == 16 << 20
    N = 64
    W = cap // (16 * N * N) + 1  # one walker more than the array holds
    rc = capi.lib().sfq_mixed_density_matrix_noalloc(ctypes.c_void_p(16), 0, ctypes.c_void_p(16),
                                                     ctypes.c_void_p(16), ctypes.c_void_p(16), int(W), 128, N, None)
    assert rc == 9  # SFQ_ERR_WORKSPACE, returned before any device work
    assert b"exceeds" in capi.lib().sfq_last_error()
