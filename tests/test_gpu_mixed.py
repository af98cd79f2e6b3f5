"""tcgen05 split-BF16 GEMM against an FP64 product (torch matmul on the same device).

Tolerances (max-norm error relative to max|C| on these random operands): 2 planes (~16
significant bits per operand) 5e-5; 3 planes 3e-5 -- the third plane adds little because the
tensor-core FP32 accumulation itself loses ~1e-7 per 16-wide accumulation step, ~1.5e-5 at
K = 2400; 1 plane 1e-2.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from safire_b200 import capi  # noqa: E402


def _run(M, N, K, batch, ab, bb, nplanes, tile_n=0, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(batch if ab else 1, M, K, generator=g, device="cuda", dtype=torch.float64)
    B = torch.randn(batch if bb else 1, N, K, generator=g, device="cuda", dtype=torch.float64)
    C = torch.full((batch, M, N), float("nan"), device="cuda", dtype=torch.float32)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(capi.lib().sfq_gemm_split_bf16(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, batch, int(ab),
                                              int(bb), nplanes, tile_n, st))
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
def test_split_bf16_gemm_two_planes(shape):
    M, N, K, batch, ab, bb, tn = shape
    assert _run(M, N, K, batch, ab, bb, 2, tn) < 5e-5


@pytest.mark.parametrize("shape", [
    (256, 256, 256, 1, 0, 0, 0),
    (200, 100, 136, 1, 0, 0, 0),
    (100, 800, 800, 3, 1, 1, 128),
    (130, 64, 512, 2, 0, 1, 64),
    (512, 1000, 2400, 1, 0, 0, 128),
])
def test_split_bf16_gemm_three_planes(shape):
    M, N, K, batch, ab, bb, tn = shape
    assert _run(M, N, K, batch, ab, bb, 3, tn) < 3e-5


def test_split_bf16_gemm_one_plane():
    assert _run(256, 384, 512, 1, 0, 0, 1) < 1e-2


def test_split_bf16_gemm_rejects_bad_k():
    rc = capi.lib().sfq_gemm_split_bf16(ctypes.c_void_p(256), ctypes.c_void_p(256), ctypes.c_void_p(256), 8, 8, 12,
                                        1, 0, 0, 3, 0, None)
    assert rc == 1


# ---------------------------------------------------------------- the mixed-precision engine
from oracle import afqmc_oracle as O  # noqa: E402
from safire_b200 import afqmc, synthetic  # noqa: E402

# per-quantity tolerances after one step against the FP64 oracle (max-norm, relative to the
# largest element), for 2 and 3 bf16 planes per operand
STEP_TOL = {capi.PRECISION_MIXED: 2e-4, capi.PRECISION_MIXED_FP32: 2e-5}


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("prec", [capi.PRECISION_MIXED, capi.PRECISION_MIXED_FP32])
@pytest.mark.parametrize("spec", [synthetic.CFG_SMALL, synthetic.CFG_MEDIUM])
def test_mixed_engine_one_step_vs_oracle(prec, spec):
    s = synthetic.make_system(spec)
    W = 16
    dt = 0.005
    eng = afqmc.AfqmcEngine(s, W, dt=dt, seed=3, precision=prec)
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    prop = O.Propagator(ham, dt, seed=3)
    wo = O.Walkers(s.initial_walkers(W))
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    tol = STEP_TOL[prec]
    # the initial energy: E1 in FP64, the exchange tensor from split-BF16 products
    assert abs(Esh - Esh_o) < tol * abs(Esh_o)
    dbg = prop.propagate(wo, Esh_o, 0)
    eng.propagate(Esh, 0)
    tol = STEP_TOL[prec]
    X = eng.fetch("X", (W, s.Nc), np.complex128)
    assert _rel(X, dbg["X"]) < tol  # fields carry the force bias from the split vbias product
    SM, pr = eng.walkers()
    assert _rel(SM, wo.SM) < tol
    assert _rel(pr["OVLP"], wo.ovlp) < 10 * tol
    assert _rel(pr["WEIGHT"], wo.weight) < 10 * tol
    # the local energy of these walkers against the oracle's on the same walkers: E1 exact (FP64),
    # exchange and Coulomb within the product tolerance
    E = eng.energy()
    Eo, _ = O.wfn_energy_noupdate(ham, O.Walkers(SM))
    assert _rel(E[:, 0], Eo[:, 0]) < 1e-10
    assert _rel(E, Eo) < tol
    eng.close()


def test_mixed_engine_rejects_unsupported_shapes():
    s = synthetic.make_system(synthetic.SystemSpec(M=20, N=5, Nc=40, decay=20.0))
    with pytest.raises(capi.SafireError, match="UNSUPPORTED"):
        afqmc.AfqmcEngine(s, 4, precision=capi.PRECISION_MIXED)


def test_mixed_engine_full_vhs_path_for_asymmetric_vectors():
    """Asymmetric Cholesky vectors: the mixed engine falls back to the full M*M vHS product."""
    s = synthetic.make_system(synthetic.CFG_SMALL)
    s.Likn = s.Likn.copy()
    s.Likn[2, 0, :] -= 2e-3
    W = 8
    eng = afqmc.AfqmcEngine(s, W, dt=0.005, seed=4, precision=capi.PRECISION_MIXED)
    assert eng.info().vhs_packed == 0
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    prop = O.Propagator(ham, 0.005, seed=4)
    wo = O.Walkers(s.initial_walkers(W))
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    prop.propagate(wo, Esh_o, 0)
    eng.propagate(Esh, 0)
    SM, pr = eng.walkers()
    assert _rel(SM, wo.SM) < STEP_TOL[capi.PRECISION_MIXED]
    eng.close()
