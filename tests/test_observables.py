"""The oracle's TwoRDM, SpinCorr and PairCorr (Observables/twordm.hpp, spincorr.hpp, paircorr.hpp),
pinned where the reference's recorded runs reach them: through the diagonal two-body and one-body
RDMs of the same estimator (which the oracle reproduces from the reference's seeded snapshots).

* TwoRDM[(a,a,a,a)][i][i][j][j] and TwoRDM[(a,a,b,b)][i][i][j][j] are the diagonal two-body RDM's
  blocks; contracting TwoRDM over its last pair gives (N_s - 1) times the one-body RDM within a
  spin and N_other times it across (each walker's mixed G is idempotent with trace N_s; with a
  multi-determinant trial each reference's G is, and the references' coefficients sum to one).
* SpinCorr's Z channel off the diagonal is a combination of the diagonal two-body RDM's blocks:
  CLOSED  -(1/2) (D_ab - D_aa)[i][j];  COLLINEAR  (1/4) (D_aa + D_bb - D_ab - D_ab^T)[i][j].
* PairCorr has no such link; it is pinned only by restating paircorr.hpp term by term, and the
  GPU tests hold the engine to this restatement.
"""
import numpy as np
import pytest

from oracle import afqmc_oracle as O
from tests.golden_io import oracle_hamiltonian, snapshot

STEPS = 4


def _run(case, observables):
    snap = snapshot(case)
    st = snap["settings"]
    ham = oracle_hamiltonian(snap)
    _, _, series = O.run_seeded(ham, 8, st["dt"], STEPS, st["seed"], ortho_interval=2, pop_interval=2,
                                measure_interval=2, mixed_interval=2, observables=observables)
    return ham, series


def _unfold(diag, M, wt):
    """The folded diagonal two-body RDM back to its blocks (diagonal_twordm.hpp:104-140)."""
    nb = 3 if wt == "COLLINEAR" else 2
    D = np.zeros((nb, M, M), np.complex128)
    it = iter(diag)
    for i in range(M):
        for j in range(i + 1, M):
            D[0, i, j] = D[0, j, i] = next(it)
        for j in range(M):
            D[1, i, j] = next(it)
    if wt == "COLLINEAR":
        for i in range(M):
            for j in range(i + 1, M):
                D[2, i, j] = D[2, j, i] = next(it)
    return D


@pytest.mark.parametrize("case,wt,nel", [("bh_rhf_closed", "CLOSED", (3, 3)), ("li_rohf_collinear", "COLLINEAR", (3, 0)),
                                         ("bh_rcasci_rhf_closed", "CLOSED", (3, 3)),
                                         ("bh_rcasci_uhf_collinear", "COLLINEAR", (3, 3))])
def test_two_rdm_and_spin_corr_follow_the_diagonal_and_one_body_rdms(case, wt, nel):
    ham, series = _run(case, dict(two_rdm=True, spin_corr=True))
    M = ham.M
    for one, diag, two, spin in zip(series["MixedEstimator/OneRDM"], series["MixedEstimator/DiagonalTwoRDM"],
                                    series["MixedEstimator/TwoRDM"], series["MixedEstimator/SpinCorr"]):
        D = _unfold(diag, M, wt)
        ii = np.arange(M)
        for b in range(D.shape[0]):
            diag_b = two[b][ii[:, None], ii[:, None], ii[None, :], ii[None, :]]
            off = ~np.eye(M, dtype=bool)
            if b != 1:  # the same-spin blocks' folded entries cover i != j
                assert np.allclose(diag_b[off], D[b][off], atol=1e-12)
            else:
                assert np.allclose(diag_b, D[1], atol=1e-12)
        up, dn = (one[0], one[1]) if wt == "COLLINEAR" else (one[0], one[0])
        assert np.allclose(np.einsum('ikjj->ik', two[0]), (nel[0] - 1) * up, atol=1e-10)
        assert np.allclose(np.einsum('ikjj->ik', two[1]), nel[1] * up, atol=1e-10)
        if wt == "COLLINEAR":
            assert np.allclose(np.einsum('ikjj->ik', two[2]), (nel[1] - 1) * dn, atol=1e-10)
        idx = 0
        for i in range(M):
            for j in range(i, M):
                if j > i:
                    if wt == "CLOSED":
                        z = -0.5 * (D[1, i, j] - D[0, i, j])
                    else:
                        z = 0.25 * (D[0, i, j] + D[2, i, j] - D[1, i, j] - D[1, j, i])
                    assert abs(spin[1, idx] - z) < 1e-12
                idx += 1


def test_pair_corr_is_refused_for_closed_walkers_and_measured_for_collinear():
    M = 14
    maps = np.array([[(i + 1) % M if i % 3 != 2 else -1 for i in range(M)], [M - 1 - i for i in range(M)]])
    _, series = _run("li_rohf_collinear", dict(two_rdm=False, spin_corr=False, pair_maps=maps))
    P = series["MixedEstimator/PairCorr"][0]
    assert P.shape == (2, 2, M, M)
    assert np.all(P[:, :, np.tril_indices(M)[0], np.tril_indices(M)[1]] == 0)  # j > i only
    assert np.all(P[0, :, 2::3, :] == 0)  # orbitals without a partner
    ham, series = _run("bh_rhf_closed", dict(two_rdm=False, spin_corr=False, pair_maps=maps[:, :5]))
    assert "MixedEstimator/PairCorr" not in series
