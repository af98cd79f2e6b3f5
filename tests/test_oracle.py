"""The oracle pinned against the reference's own known-answer vectors and invariants.

KATs come from tests/test_sdet_ops.cpp of the reference (extracted by
tests/golden/make_sdet_kats.py); the comparison tolerance is the reference's own
utils::Approx default (atol = rtol = 1e-8, tests/test_common.hpp:383-444).
"""
import math

import numpy as np
import pytest

from golden_io import sdet_kats
from oracle import afqmc_oracle as O
from oracle import philox
from safire_b200 import synthetic

TOL = 1e-8


def approx(a, b, tol=TOL):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b)))


@pytest.fixture(scope="module")
def kats():
    return sdet_kats()


def _batch(m, nw=5):
    return np.broadcast_to(m, (nw,) + m.shape).copy()


def test_log_overlap_kat(kats):
    A, B = kats["m_a"], _batch(kats["m_b"])
    ov = O.log_overlap(A, B)
    assert approx(ov, np.log(kats["ov_base_log_of"]))
    # sub-block views: A(0:2, 0:3), B(:, 0:3, 0:2)
    ov2 = O.log_overlap(A[:2, :3], B[:, :3, :2])
    assert approx(ov2, np.log(kats["ov2_base_log_of"]))


def test_mixed_density_matrix_kat(kats):
    A, B = kats["m_a"], _batch(kats["m_b"])
    G, ov = O.mixed_density_matrix(A, B, compact=False)
    assert approx(G, _batch(kats["v_ref"]))
    assert approx(ov, np.log(kats["ov_base_log_of"]))
    Gc, ov = O.mixed_density_matrix(A, B, compact=True)
    assert approx(Gc, _batch(kats["vc_ref"]))
    G2, _ = O.mixed_density_matrix(A[:2, :3], B[:, :3, :2], compact=False)
    assert approx(G2, _batch(kats["v_ref_2"]))
    Gc2, _ = O.mixed_density_matrix(A[:2, :3], B[:, :3, :2], compact=True)
    assert approx(Gc2, _batch(kats["vc_ref_2"]))


def test_inverse_logdet_kat(kats):
    inv, ld = O.inverse_logdet(_batch(kats["inv_m_a"]))
    assert approx(inv, _batch(kats["inv_ref"]))
    assert approx(ld, kats["logdetA_ref"])


def test_lu_solve_kat(kats):
    A, B = kats["ma_lu"], kats["mb_lu"]
    ld, inv = O.lu_logdet_inverse(A)
    assert approx(inv @ B, kats["xv_ref"])
    assert approx(ld, kats["ovlp_lu_ref"])


def test_orthogonalize_kat(kats):
    # test_sdet_ops.cpp:294-304: Log_Overlap(Q, Q) == 0 after orthogonalize
    Q, _ = O.orthogonalize(_batch(kats["m_b"]))
    ov = O.log_overlap(np.conj(Q[0].T), Q)
    assert np.max(np.abs(ov)) < 1e-12
    # R has a positive real diagonal after the sign fix: Q^H B is upper triangular, Re diag > 0
    R = np.conj(Q[0].T) @ kats["m_b"]
    assert np.all(np.diag(R).real > 0)
    assert np.max(np.abs(np.tril(R, -1))) < 1e-12


def test_singular_overlap_gives_zero_inverse():
    # getri_or_zero (nda_functions.hpp:422-438): a singular T yields a zero inverse
    T = np.zeros((3, 3), np.complex128)
    T[0, 0] = 1.0
    ld, inv = O.lu_logdet_inverse(T)
    assert np.all(inv == 0)
    assert ld.real < -700   # log(tiny) of the zero pivots


def test_philox_known_answers():
    # Random123 philox4x32_10 KATs
    r = philox.philox4x32_10(0, 0, 0, 0, 0, 0)
    assert [int(x) for x in r] == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    r = philox.philox4x32_10(0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344, 0xa4093822, 0x299f31d0)
    assert [int(x) for x in r] == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]
    u = philox.uniforms(0, philox.STREAM_FIELDS, 7, 5, 9)
    assert u.shape == (5, 9) and np.all(u > 0) and np.all(u < 1)


def test_probit_values():
    p = np.array([1e-6, 0.01, 0.3, 0.5, 0.7, 0.99, 1 - 1e-6])
    from scipy.special import ndtri
    assert np.max(np.abs(O.probit(p) - ndtri(p)) / np.maximum(1, np.abs(ndtri(p)))) < 1.2e-9 * 5
    assert O.probit(np.array([0.0]))[0] == -np.inf


@pytest.fixture(scope="module")
def small():
    s = synthetic.make_system(synthetic.CFG_SMALL)
    return s, O.Hamiltonian(s.hcore, s.Likn, s.PsiT)


def test_trial_invariants(small):
    s, ham = small
    G = O.trial_density(ham)[0]
    # full G_MF = PsiT^T G: trace N, Hermitian
    Gf = ham.PsiT.T @ G
    assert abs(np.trace(Gf) - ham.N) < 1e-12
    assert np.max(np.abs(Gf - np.conj(Gf.T))) < 1e-12


def test_trial_energy_closed_form(small):
    # E(trial) = 2 sum_occ h_aa + sum_n [2 (tr L_n^occ)^2 - sum_ab (L_n^occ)_ab^2]
    s, ham = small
    W = O.Walkers(s.initial_walkers(2))
    O.wfn_energy(ham, W)
    P = np.real(ham.PsiT)
    e1 = 2 * np.trace(P @ s.hcore @ P.T)
    Locc = np.einsum('ai,ikn,bk->nab', P, s.Likn, P)
    ej = 2 * np.sum(np.einsum('naa->n', Locc) ** 2)
    exx = -np.sum(Locc * Locc)
    assert abs(W.e1[0] - e1) < 1e-10 * abs(e1)
    assert abs(W.ej[0] - ej) < 1e-10 * abs(ej)
    assert abs(W.exx[0] - exx) < 1e-10 * abs(exx)


def test_taylor_matches_exponential(small):
    from scipy.linalg import expm
    rng = np.random.default_rng(1)
    M, N = 8, 3
    V = rng.normal(size=(2, M, M)) * 1e-3
    V = V + np.transpose(V, (0, 2, 1))
    S = rng.normal(size=(2, M, N)) + 1j * rng.normal(size=(2, M, N))
    out = O.apply_expM(V.astype(np.complex128), S, order=6)
    ref = np.stack([expm(1j * V[i]) @ S[i] for i in range(2)])
    assert np.max(np.abs(out - ref)) < 1e-14 * 10


def test_orthogonalize_preserves_G(small):
    s, ham = small
    rng = np.random.default_rng(2)
    Wk = s.initial_walkers(3) + 0.1 * (rng.normal(size=(3, s.M, s.N)) + 1j * rng.normal(size=(3, s.M, s.N)))
    G0, _ = O.mixed_density_matrix(ham.PsiT, Wk)
    Q, _ = O.orthogonalize(Wk)
    G1, _ = O.mixed_density_matrix(ham.PsiT, Q)
    assert np.max(np.abs(G0 - G1)) < 1e-12


def test_comb_conserves_population():
    rng = np.random.default_rng(3)
    for _ in range(20):
        w = rng.exponential(size=37)
        w[rng.integers(0, 37, 5)] = 0.0
        off = O.comb(w, rng.uniform(), 37)
        assert off.sum() == 37
        assert np.all(off[w == 0] == 0)
        plan = O.copy_plan(off)
        assert len(plan) == int(np.sum(off == 0))


def test_small_run_is_deterministic(small):
    s, ham = small
    res = []
    for _ in range(2):
        W = O.Walkers(s.initial_walkers(8))
        Esh = O.init_walkers(ham, W)
        prop = O.Propagator(ham, 0.005, seed=0)
        Esh, _ = O.run(ham, W, prop, 12, Esh, ortho_interval=5, pop_interval=10)
        res.append((Esh, W.weight.copy(), W.SM.copy()))
    assert res[0][0] == res[1][0]
    assert np.array_equal(res[0][1], res[1][1])
    assert np.array_equal(res[0][2], res[1][2])
