"""The exact-accumulation tensor-core products (int8 fixed-point slices, tcgen05 kind::i8).

* The products are bit-identical to the numpy restatement of their arithmetic (tests/islice_ref.py):
  the slices and the int32 group sums are exact and the FP64 combination rounds once to FP32, so
  there is nothing to tolerate.
* They carry no accumulation bias: on positive data the split-BF16 product of the same operands
  comes out shrunk (the tensor cores' FP32 accumulation rounds toward zero), this one does not.
* The INT8X3 engine against the FP64 oracle after one step and on the local energy of identical
  walkers, at tolerances set by 3 slices (2^-24 of each row's largest entry).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from safire_b200 import capi  # noqa: E402
from tests import islice_ref as R  # noqa: E402


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _int8_gemm(A, B, ns, bn=0, ks=1):
    M, K = A.shape
    N = B.shape[0]
    C = torch.full((ks, M, N), float("nan"), dtype=torch.float32, device="cuda")
    dA, dB = _dev(A), _dev(B)
    capi.check(capi.lib().sfq_gemm_int8_slices(dA.data_ptr(), dB.data_ptr(), C.data_ptr(), M, N, K, ns, bn, ks, None))
    torch.cuda.synchronize()
    return C.cpu().numpy()


def _operands(M, N, K, seed):
    """rows of very different scales, a zero row, a row with one large entry"""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-3, 3, (M, 1))
    B = rng.standard_normal((N, K)) * 10.0 ** rng.uniform(-2, 2, (N, 1))
    A[1] = 0.0
    A[2, 5 % K] = 1e4
    B[3] = np.abs(B[3])
    return A, B


@pytest.mark.parametrize("ns", [2, 3])
@pytest.mark.parametrize("K,bn", [(70, 64), (400, 128), (400, 160), (2400, 160), (1000, 64)])
def test_int8_slice_product_is_bit_exact(ns, K, bn):
    A, B = _operands(300, 250, K, seed=K + bn + ns)
    C = _int8_gemm(A, B, ns, bn)[0]
    ref = R.gemm(A, B, ns)
    assert np.array_equal(C, ref), np.max(np.abs(C - ref))
    # and it is the product: within the slices' resolution of the FP64 one
    exact = A @ B.T
    scale = np.max(np.abs(A), axis=1)[:, None] * np.max(np.abs(B), axis=1)[None, :] * K
    tol = 2.0 ** (-20 if ns == 3 else -12)
    assert np.all(np.abs(C - exact) <= tol * scale + 1e-6 * np.abs(exact))


def test_int8_slice_product_k_split_partials():
    """K split into ranges of whole 128-element blocks (at either K slice width of the kernel): each
    partial product is the exact product over its range."""
    A, B = _operands(200, 170, 2400, seed=11)
    for ks in (5, 2):  # 480 and 1200 elements per range: 64- and 128-element K slices
        C = _int8_gemm(A, B, 3, 160, ks)
        KT = (2400 + 127) // 128
        for s in range(ks):
            k0, k1 = 128 * (KT * s // ks), min(2400, 128 * (KT * (s + 1) // ks))
            assert np.array_equal(C[s], R.gemm(A, B, 3, k0=k0, k1=k1)), (ks, s)


def test_int8_slices_carry_no_accumulation_bias():
    """Positive operands, K = 2400: the split-BF16 product (3 planes, FP32 accumulation rounding toward
    zero) comes out smaller than the exact one by ~1e-5 relative, every element the same way; the
    int8-slice product's errors are the slices' round-to-nearest ones, mean zero."""
    rng = np.random.default_rng(5)
    A = rng.uniform(0.5, 1.0, (256, 2400))
    B = rng.uniform(0.5, 1.0, (256, 2400))
    exact = A @ B.T
    C = _int8_gemm(A, B, 3, 128)[0]
    rel = (C.astype(np.float64) - exact) / exact
    assert abs(np.mean(rel)) < 2e-9, np.mean(rel)
    Cb = torch.empty((256, 256), dtype=torch.float32, device="cuda")
    dA, dB = _dev(A), _dev(B)
    capi.check(capi.lib().sfq_gemm_split_bf16(dA.data_ptr(), dB.data_ptr(), Cb.data_ptr(), 256, 256, 2400, 1, 0, 0, 3,
                                              128, None))
    torch.cuda.synchronize()
    relb = (Cb.cpu().numpy().astype(np.float64) - exact) / exact
    assert np.mean(relb) < -1e-6  # the bias the int8 slices remove


@pytest.mark.parametrize("W,M,N,half", [(3, 100, 20, 32), (3, 100, 20, 64), (2, 160, 17, 80), (4, 19, 3, 32),
                                        (2, 400, 100, 80)])
def test_int8_taylor_product_is_bit_exact(W, M, N, half):
    rng = np.random.default_rng(M + N)
    A = (rng.standard_normal((W, N, M)) + 1j * rng.standard_normal((W, N, M))) * 10.0 ** rng.uniform(-2, 2, (W, N, 1))
    V = rng.standard_normal((W, M, M)) + 1j * rng.standard_normal((W, M, M))
    V[0, 2] *= 1e-3
    C = torch.full((2, W, N, M), float("nan"), dtype=torch.float32, device="cuda")
    dA, dV = _dev(A), _dev(V)
    capi.check(capi.lib().sfq_gemm_int8_cplx_b(dA.data_ptr(), dV.data_ptr(), C.data_ptr(), W, M, N, 3, half, None))
    torch.cuda.synchronize()
    got = C.cpu().numpy()
    ref = R.cplx_b(A, V, 3)
    assert np.array_equal(got, ref), np.max(np.abs(got - ref))
    exact = np.einsum("wai,wji->waj", A, V)
    assert np.max(np.abs(got[0] + 1j * got[1] - exact)) < 1e-6 * np.max(np.abs(exact))


def test_int8_product_rejects_bad_arguments():
    L = capi.lib()
    p = ctypes.c_void_p(256)
    assert L.sfq_gemm_int8_slices(p, p, p, 8, 8, 16, 4, 0, 1, None) == 2    # slices
    assert L.sfq_gemm_int8_slices(p, p, p, 8, 8, 16, 3, 96, 1, None) == 2   # tile width not built
    assert L.sfq_gemm_int8_cplx_b(p, p, p, 1, 16, 4, 3, 48, None) == 2      # half not built


# ---------------------------------------------------------------- the INT8X3 engine
from oracle import afqmc_oracle as O  # noqa: E402
from safire_b200 import afqmc, synthetic  # noqa: E402


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("spec", [synthetic.CFG_SMALL, synthetic.CFG_MEDIUM,
                                  synthetic.SystemSpec(M=19, N=3, Nc=78, decay=19.0)])
def test_int8x3_engine_one_step_vs_oracle(spec):
    """One step of the INT8X3 engine against the FP64 oracle: fields, walkers, overlaps, weights and
    the local energies of the propagated walkers; any nmo and nchol (19 and 78 here, BH's sizes).
    The bounds are those of 3 slices, 2^-24 of each row's largest entry: rows dominated by one entry
    (the trial's near-unit orbitals, the first energy) carry their other entries to ~1e-7 absolute."""
    s = synthetic.make_system(spec)
    W = 16
    dt = 0.005
    eng = afqmc.AfqmcEngine(s, W, dt=dt, seed=3, precision=capi.PRECISION_INT8X3)
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    prop = O.Propagator(ham, dt, seed=3)
    wo = O.Walkers(s.initial_walkers(W))
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    assert abs(Esh - Esh_o) < 5e-6 * abs(Esh_o)
    dbg = prop.propagate(wo, Esh_o, 0)
    eng.propagate(Esh, 0)
    X = eng.fetch("X", (W, s.Nc), np.complex128)
    assert _rel(X, dbg["X"]) < 1e-6
    SM, pr = eng.walkers()
    assert _rel(SM, wo.SM) < 2e-6
    assert _rel(pr["OVLP"], wo.ovlp) < 5e-6
    assert _rel(pr["WEIGHT"], wo.weight) < 2e-5
    E = eng.energy()
    Eo, _ = O.wfn_energy_noupdate(ham, O.Walkers(SM))
    assert _rel(E[:, 0], Eo[:, 0]) < 1e-10
    assert _rel(E, Eo) < 2e-6
    eng.close()


@pytest.mark.parametrize("spec", [synthetic.CFG_SMALL, synthetic.SystemSpec(M=19, N=3, Nc=78, decay=19.0)])
def test_int8x3_complex_trial_one_step_vs_oracle(spec):
    """A complex trial (the orbitals given phases e^{i theta_j}): Lnak is complex, so the force bias and
    the exchange tensor are completed by the products with its imaginary rows (accumulated into the
    same outputs).  One step against the FP64 oracle at the closed-shell test's bounds."""
    s = synthetic.make_system(spec)
    s.PsiT = s.PsiT * np.exp(1j * np.linspace(0.0, 1.0, s.M))[None, :]
    W, dt = 16, 0.005
    eng = afqmc.AfqmcEngine(s, W, dt=dt, seed=3, precision=capi.PRECISION_INT8X3)
    assert eng.info().lnak_complex == 1
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    prop = O.Propagator(ham, dt, seed=3)
    wo = O.Walkers(s.initial_walkers(W))
    Esh_o = O.init_walkers(ham, wo)
    Esh = eng.init()
    assert abs(Esh - Esh_o) < 5e-6 * abs(Esh_o)
    dbg = prop.propagate(wo, Esh_o, 0)
    eng.propagate(Esh, 0)
    X = eng.fetch("X", (W, s.Nc), np.complex128)
    assert _rel(X, dbg["X"]) < 1e-6
    SM, pr = eng.walkers()
    assert _rel(SM, wo.SM) < 2e-6
    assert _rel(pr["OVLP"], wo.ovlp) < 5e-6
    assert _rel(pr["WEIGHT"], wo.weight) < 2e-5
    E = eng.energy()
    Eo, _ = O.wfn_energy_noupdate(ham, O.Walkers(SM))
    assert _rel(E[:, 0], Eo[:, 0]) < 1e-10
    assert _rel(E, Eo) < 2e-6
    eng.close()


def test_int8x3_collinear_walkers_vs_fp64_engine():
    """COLLINEAR walkers (the reference's Li ROHF fixture, M=14, 2 up + 1 down, Nc=70) in INT8X3
    against the FP64 engine, which reproduces the reference's recorded Li runs: the trial's energy,
    the energies of identical walkers (same-spin exchange, per-spin Coulomb) and one step from
    identical walkers and seeded fields, at the 3-slice bounds of the closed-shell test."""
    from tests.golden_io import engine_system, snapshot
    s = engine_system(snapshot("li_rohf_collinear"))
    W, dt = 32, 0.01
    e64 = afqmc.AfqmcEngine(s, W, dt=dt, seed=5, precision=capi.PRECISION_FP64)
    e8 = afqmc.AfqmcEngine(s, W, dt=dt, seed=5, precision=capi.PRECISION_INT8X3)
    E64, E8 = e64.init(), e8.init()
    assert abs(E8 - E64) < 2e-6 * abs(E64)
    for st in range(3):  # walkers away from the trial
        e64.propagate(E64, st)
    SM, pr = e64.walkers()
    e8.set_walkers(SM, pr)
    assert _rel(e8.energy(), e64.energy()) < 2e-6
    e64.propagate(E64, 7)
    e8.propagate(E64, 7)
    X8, X64 = (e.fetch("X", (W, s.Nc), np.complex128) for e in (e8, e64))
    assert _rel(X8, X64) < 1e-6
    S8, p8 = e8.walkers()
    S64, p64 = e64.walkers()
    assert _rel(S8, S64) < 2e-6
    assert _rel(p8["OVLP"], p64["OVLP"]) < 5e-6
    assert _rel(p8["WEIGHT"], p64["WEIGHT"]) < 2e-5
    e64.close()
    e8.close()


@pytest.mark.parametrize("case", ["bh_ghf_noncollinear", "bh_uhf_noncollinear"])
def test_int8x3_noncollinear_walkers_vs_fp64_engine(case):
    """NONCOLLINEAR walkers (the reference's BH spinor fixtures, M=19 in 2M=38 spinor rows, N=6,
    Nc=78; the GHF trial mixes the components) in INT8X3 against the FP64 engine, which reproduces
    the reference's recorded runs: the trial's energy, the energies of identical walkers, and three
    steps from identical walkers and seeded fields, at the 3-slice bounds of the closed-shell test."""
    from tests.golden_io import engine_system, snapshot
    s = engine_system(snapshot(case))
    W, dt = 32, 0.01
    e64 = afqmc.AfqmcEngine(s, W, dt=dt, seed=5, precision=capi.PRECISION_FP64)
    e8 = afqmc.AfqmcEngine(s, W, dt=dt, seed=5, precision=capi.PRECISION_INT8X3)
    E64, E8 = e64.init(), e8.init()
    assert abs(E8 - E64) < 2e-6 * abs(E64)
    for st in range(3):  # walkers away from the trial
        e64.propagate(E64, st)
    SM, pr = e64.walkers()
    assert SM.shape == (W, 2 * s.M, s.N)
    e8.set_walkers(SM, pr)
    assert _rel(e8.energy(), e64.energy()) < 2e-6
    for st in (7, 8, 9):
        e64.propagate(E64, st)
        e8.propagate(E64, st)
        X8, X64 = (e.fetch("X", (W, s.Nc), np.complex128) for e in (e8, e64))
        assert _rel(X8, X64) < 1e-6 * (st - 6)
    S8, p8 = e8.walkers()
    S64, p64 = e64.walkers()
    assert _rel(S8, S64) < 6e-6
    assert _rel(p8["OVLP"], p64["OVLP"]) < 1.5e-5
    assert _rel(p8["WEIGHT"], p64["WEIGHT"]) < 6e-5
    assert _rel(e8.energy(), e64.energy()) < 2e-6
    e64.close()
    e8.close()


@pytest.mark.parametrize("case,phased", [("bh_rcasci_rhf_closed", False), ("bh_rcasci_uhf_collinear", False),
                                         ("bh_rcasci_ghf_noncollinear", False), ("bh_rcasci_rhf_closed", True)])
def test_int8x3_multi_determinant_trials_vs_fp64_engine(case, phased):
    """Multi-determinant NOMSD trials (the reference's BH CASCI fixtures, 34 determinants; CLOSED,
    COLLINEAR and NONCOLLINEAR walkers) in INT8X3 against the FP64 engine, which reproduces the
    reference's recorded CASCI runs: the force bias from the ci-weighted full G minus the trial's,
    sliced against L over (i, k); every determinant's exchange from its own slices.  The trial's
    energy, the energies of identical walkers and three steps from identical walkers and seeded
    fields, at the bounds of the single-determinant tests.  Phased: every determinant's orbitals given
    phases e^{i theta_j}, a complex trial (complex Lnak per determinant)."""
    from tests.golden_io import engine_system, snapshot
    s = engine_system(snapshot(case))
    if phased:
        s.PsiT = s.PsiT * np.exp(1j * np.linspace(0.0, 1.0, s.PsiT.shape[-1]))
    W, dt = 32, 0.01
    e64 = afqmc.AfqmcEngine(s, W, dt=dt, seed=5, precision=capi.PRECISION_FP64)
    e8 = afqmc.AfqmcEngine(s, W, dt=dt, seed=5, precision=capi.PRECISION_INT8X3)
    E64, E8 = e64.init(), e8.init()
    assert abs(E8 - E64) < 2e-6 * abs(E64)
    for st in range(3):  # walkers away from the trial
        e64.propagate(E64, st)
    SM, pr = e64.walkers()
    e8.set_walkers(SM, pr)
    assert _rel(e8.energy(), e64.energy()) < 2e-6
    for st in (7, 8, 9):
        e64.propagate(E64, st)
        e8.propagate(E64, st)
        X8, X64 = (e.fetch("X", (W, s.Nc), np.complex128) for e in (e8, e64))
        assert _rel(X8, X64) < 1e-6 * (st - 6)
    S8, p8 = e8.walkers()
    S64, p64 = e64.walkers()
    assert _rel(S8, S64) < 6e-6
    assert _rel(p8["OVLP"], p64["OVLP"]) < 1.5e-5
    assert _rel(p8["WEIGHT"], p64["WEIGHT"]) < 6e-5
    assert _rel(e8.energy(), e64.energy()) < 2e-6
    e64.close()
    e8.close()


def test_bounded_waits_expire_and_report_timeout():
    """The product's loads are held back by a flag nothing sets and every wait is limited to 1 ms:
    each wait expires, the kernel reports SFQ_ERR_TIMEOUT with nothing in flight and its tensor
    memory freed, and the next product on the same context runs and is exact."""
    L = capi.lib()
    assert L.sfq_selftest_wait_expiry(1_000_000, None) == 8  # SFQ_ERR_TIMEOUT
    A, B = _operands(200, 150, 400, seed=9)
    assert np.array_equal(_int8_gemm(A, B, 3, 128)[0], R.gemm(A, B, 3))
    assert L.sfq_selftest_wait_expiry(0, None) == 2  # no limit is no test
