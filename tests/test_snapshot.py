"""The reference's seeded snapshot of a real molecule, replayed on its own random streams.

The dense-Cholesky NOMSD cases of the reference's functional tests (BH and Li; CLOSED, COLLINEAR and
NONCOLLINEAR walkers; single-determinant and 34-determinant CASCI trials; seed 42, 50 walkers,
20 steps, one rank) recorded every energy-estimator observable; the reference's runner requires a
rerun to reproduce them to 1e-9.
These tests pin:

  * the host random streams (std::mt19937 via split_seed, uniform_real_distribution) against the
    C++ standard's known answer and numpy's independent MT19937;
  * the oracle's whole stage -- vbias, fields, vHS, P1 * Taylor * P1, overlaps, walker update,
    orthogonalization, comb, energies and the estimator -- against the recorded snapshot;
  * the HDF5 reader and the input loaders against the reference's own files, where those are
    present (they are only read when the fixture is regenerated).
"""
import os

import numpy as np
import pytest

from oracle import afqmc_oracle as O
from oracle.mt19937 import MT19937, HostRandomGenerator, split_seed
from tests.golden_io import SNAPSHOT_OBSERVABLES, bh_snapshot, oracle_hamiltonian, snapshot, snapshot_match

# the SAFIRE source tree, when present on this machine (only then are its own input files read)
REF_ROOT = os.environ.get("SAFIRE_REFERENCE_ROOT", "")
REF = os.path.join(REF_ROOT, "tests", "functional") if REF_ROOT else ""


def test_mt19937_known_answers():
    # C++ [rand.predef]: the 10000th consecutive invocation of a default-constructed mt19937 produces 4123659995
    assert MT19937().raw(10000)[-1] == 4123659995
    for seed in (0, 42, split_seed(42, 0, 1)):
        a = MT19937(seed).raw(1500).astype(np.uint64)
        b = np.random.RandomState(seed & 0xFFFFFFFF).randint(0, 2**32, size=1500, dtype=np.uint64)
        assert np.array_equal(a, b)


def test_uniforms_from_two_draws():
    g, h = HostRandomGenerator(7), MT19937(7)
    u = g.uniforms(1000)
    r = h.raw(2000).astype(np.float64).reshape(-1, 2)
    assert np.array_equal(u, (r[:, 0] + r[:, 1] * 2.0**32) / 2.0**64)
    assert np.all((u >= 0.0) & (u < 1.0))


def test_split_seed_streams_distinct():
    seeds = {split_seed(42, rank, stream) for rank in range(64) for stream in range(4)}
    assert len(seeds) == 256
    assert all(0 <= s < 2**64 for s in seeds)


def _oracle_hamiltonian(snap):
    return oracle_hamiltonian(snap)


SNAPSHOT_CASES = ["bh_rhf_closed", "bh_uhf_collinear", "bh_rhf_collinear", "li_rohf_collinear",
                  "bh_rhf_noncollinear", "bh_uhf_noncollinear", "bh_ghf_noncollinear"]
# CASCI trials of 34 determinants
MULTIDET_CASES = ["bh_rcasci_rhf_closed", "bh_rcasci_rhf_collinear", "bh_rcasci_rhf_noncollinear",
                  "bh_rcasci_uhf_collinear", "bh_rcasci_uhf_noncollinear", "bh_rcasci_ghf_noncollinear"]


@pytest.mark.parametrize("case", SNAPSHOT_CASES + MULTIDET_CASES)
def test_oracle_reproduces_reference_snapshot(case):
    """BH with an RHF trial and CLOSED walkers; COLLINEAR walkers with BH's UHF and RHF trials and Li's
    fully polarized ROHF trial (no down electrons); NONCOLLINEAR walkers with BH's RHF and UHF trials
    upgraded to spinors and a GHF trial; and 34-determinant CASCI trials with each walker type."""
    snap = snapshot(case)
    st = snap["settings"]
    assert st["num_ranks"] == 1
    ham = _oracle_hamiltonian(snap)
    _, _, series = O.run_seeded(ham, st["nwalk"], st["dt"], st["steps"], st["seed"],
                                ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                measure_interval=st["measure_interval"],
                                equilibration_steps=st["equilibration_steps"])
    for k in SNAPSHOT_OBSERVABLES:
        assert len(series[k]) == st["steps"]
        B = snapshot_match(series[k], snap["recorded"][k], O.rebinned_average)
        assert B is not None, (k, snap["recorded"][k])


def test_snapshot_detects_a_planted_mistake():
    """A field stream off by one draw, or one other seed, no longer reproduces the snapshot."""
    snap = bh_snapshot()
    st = snap["settings"]
    ham = O.Hamiltonian(snap["hcore"], snap["Likn"], snap["PsiT"], snap["E0"])
    _, _, series = O.run_seeded(ham, st["nwalk"], st["dt"], st["steps"], st["seed"] + 1,
                                ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                measure_interval=st["measure_interval"])
    assert snapshot_match(series["Energy"], snap["recorded"]["Energy"], O.rebinned_average) is None


@pytest.mark.skipif(not (REF and os.path.isdir(REF)),
                    reason="SAFIRE_REFERENCE_ROOT does not name the reference tree on this machine")
def test_loaders_read_reference_files():
    from safire_b200.h5read import H5File
    from safire_b200.inputs import InputError, load_dense_hamiltonian, load_nomsd_trial
    snap = bh_snapshot()
    wfn = load_nomsd_trial(f"{REF}/afqmc_inputs/BH/afqmc_rhf_nomsd.h5")
    ham = load_dense_hamiltonian(f"{REF}/afqmc_inputs/BH/afqmc_H_rhf_closed.h5", wfn["nup"])
    assert np.array_equal(ham["hcore"], snap["hcore"]) and np.array_equal(ham["Likn"], snap["Likn"])
    assert np.array_equal(wfn["PsiT"], snap["PsiT"]) and ham["E0"] == snap["E0"]
    f = H5File(f"{REF}/afqmc_inputs/BH/afqmc_H_rhf_closed.h5")
    assert f.keys("Hamiltonian") == ["DenseFactorized", "X", "hcore"]
    assert f.shape("Hamiltonian/DenseFactorized/L") == (1, 1, 19, 1, 19, 78)
    # what the CLOSED single-determinant dense path does not take is refused with the reason
    with pytest.raises(InputError):
        load_nomsd_trial(f"{REF}/afqmc_inputs/BH/afqmc_uhf_nomsd.h5")       # collinear trial, CLOSED walkers
    coll = load_nomsd_trial(f"{REF}/afqmc_inputs/Li/rohf_nomsd_polarized.h5", "COLLINEAR")
    li = snapshot("li_rohf_collinear")
    assert coll["ndn"] == 0 and np.array_equal(coll["PsiT_up"], li["PsiT_up"])
    up = load_nomsd_trial(f"{REF}/afqmc_inputs/BH/afqmc_rhf_nomsd.h5", "COLLINEAR")  # closed trial, upgraded
    assert np.array_equal(up["PsiT_up"], up["PsiT_dn"]) and np.array_equal(up["PsiT_up"], snap["PsiT"])
    with pytest.raises(InputError):
        load_nomsd_trial(f"{REF}/afqmc_inputs/BH/afqmc_casci_rhf_nomsd.h5")  # several determinants
    with pytest.raises(InputError):
        load_dense_hamiltonian(f"{REF}/afqmc_inputs/BH/afqmc_H_rhf_noncollinear.h5", 3)


LOAD_CASES = [("bh_rhf_closed", "BH", "afqmc_H_rhf_closed.h5", "afqmc_rhf_nomsd.h5"),
              ("bh_rhf_collinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_rhf_nomsd.h5"),
              ("bh_uhf_collinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_uhf_nomsd.h5"),
              ("bh_rhf_noncollinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_rhf_nomsd.h5"),
              ("bh_uhf_noncollinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_uhf_nomsd.h5"),
              ("bh_ghf_noncollinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_ghf_nomsd.h5"),
              ("bh_rcasci_rhf_closed", "BH", "afqmc_H_rhf_closed.h5", "afqmc_casci_rhf_nomsd.h5"),
              ("bh_rcasci_rhf_collinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_casci_rhf_nomsd.h5"),
              ("bh_rcasci_uhf_collinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_casci_uhf_nomsd.h5"),
              ("bh_rcasci_rhf_noncollinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_casci_rhf_nomsd.h5"),
              ("bh_rcasci_uhf_noncollinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_casci_uhf_nomsd.h5"),
              ("bh_rcasci_ghf_noncollinear", "BH", "afqmc_H_rhf_closed.h5", "afqmc_casci_ghf_nomsd.h5"),
              ("li_rohf_collinear", "Li", "hamil_closed.h5", "rohf_nomsd_polarized.h5")]


@pytest.mark.skipif(not (REF and os.path.isdir(REF)),
                    reason="SAFIRE_REFERENCE_ROOT does not name the reference tree on this machine")
@pytest.mark.parametrize("case,system,ham,wfn", LOAD_CASES)
def test_load_system_reads_every_walker_type_and_trial(case, system, ham, wfn):
    """load_system builds, from the reference's own input files, the same System the snapshot case's
    fixture gives the engine: CLOSED, COLLINEAR and NONCOLLINEAR walkers, single-determinant and the
    34-determinant CASCI trials, BH and Li."""
    from safire_b200.inputs import load_system
    from tests.golden_io import engine_system
    snap = snapshot(case)
    wt = snap["settings"]["walker_type"]
    got = load_system(f"{REF}/afqmc_inputs/{system}/{ham}", f"{REF}/afqmc_inputs/{system}/{wfn}", wt)
    want = engine_system(snap)
    assert (got.M, got.N, got.Nc, got.nel_dn, got.npol) == (want.M, want.N, want.Nc, want.nel_dn, want.npol)
    assert got.E0 == want.E0
    for k in ("hcore", "Likn", "PsiT"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    assert (got.ci is None) == (want.ci is None)
    if want.ci is not None:
        assert np.array_equal(got.ci, want.ci)


def test_collinear_with_identical_spins_is_closed():
    """COLLINEAR walkers whose up and down trials are the same RHF orbitals follow the CLOSED walk:
    same fields, overlaps (two equal determinants) and energies."""
    snap = bh_snapshot()
    closed = O.Hamiltonian(snap["hcore"], snap["Likn"], snap["PsiT"], snap["E0"])
    coll = O.CollinearHamiltonian(snap["hcore"], snap["Likn"], snap["PsiT"], snap["PsiT"], snap["E0"])
    runs = [O.run_seeded(h, 16, 0.01, 12, 7, ortho_interval=5, pop_interval=3, measure_interval=1)
            for h in (closed, coll)]
    assert abs(runs[0][0] - runs[1][0]) < 1e-12 * abs(runs[0][0])
    for k in ("Energy", "ExchangeEnergy", "CoulombEnergy", "Overlap"):
        a, b = np.asarray(runs[0][2][k]), np.asarray(runs[1][2][k])
        assert np.max(np.abs(a - b)) < 1e-10 * np.max(np.abs(a)), k


RDM_CASES = ["bh_rhf_closed", "bh_uhf_collinear", "bh_uhf_noncollinear", "bh_rcasci_uhf_collinear",
             "bh_rcasci_uhf_noncollinear", "li_rohf_collinear"]


@pytest.mark.parametrize("case", RDM_CASES)
def test_oracle_reproduces_recorded_rdms(case):
    """The mixed (every 2 steps) and back-propagated (2 steps, path restoration) one-body and diagonal
    two-body RDMs the reference recorded with its back-propagation cases: CLOSED, COLLINEAR,
    NONCOLLINEAR, a 34-determinant trial, Li."""
    snap = snapshot(case)
    st = snap["settings"]
    _, _, series = O.run_seeded(oracle_hamiltonian(snap), st["nwalk"], st["dt"], st["steps"], st["seed"],
                                ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                measure_interval=st["measure_interval"], mixed_interval=snap["mixed_interval"],
                                bp_steps=snap["bp_steps"], bp_ortho_interval=snap["bp_ortho_interval"])
    rdms = [k for k in snap["recorded"] if k.startswith(("MixedEstimator", "BackPropEstimator"))]
    assert len(rdms) == 4
    for k in rdms:
        assert len(series[k]) == st["steps"] // 2
        assert np.asarray(series[k]).shape[1:] == snap["recorded"][k][0].shape
        assert snapshot_match(series[k], snap["recorded"][k], O.rebinned_average) is not None, k


@pytest.mark.skipif(not (REF and os.path.isdir(REF)),
                    reason="SAFIRE_REFERENCE_ROOT does not name the reference tree on this machine")
def test_h5read_reads_every_reference_file_and_chunked_data():
    """The reader parses every HDF5 file of the reference tree (groups, datasets, attributes), and its
    chunked, deflate-compressed datasets decode to consistent data: in a recorded results file the
    back-propagated one-body RDM has the electron count as its trace in every bin."""
    import glob
    from safire_b200.h5read import H5File
    root = os.path.dirname(os.path.dirname(REF))
    files = sorted(glob.glob(os.path.join(root, "**", "*.h5"), recursive=True))
    assert len(files) > 100
    ndata = 0
    for p in files:
        f = H5File(p)
        stack = ["/"]
        while stack:
            q = stack.pop()
            for k in f.keys(q):
                path = q.rstrip("/") + "/" + k
                if f.is_group(path):
                    f.attrs(path)
                    stack.append(path)
                else:
                    f[path]
                    ndata += 1
    assert ndata > 1000
    res = os.path.join(root, "docs", "examples", "solids", "02_C_diamond_pyscf_interface", "data", "afqmc.results.h5")
    if os.path.exists(res):
        f = H5File(res)
        R = f["/Measurements/Stage0/BackPropEstimator/Steps=100/OneRDM/bins"]
        tr = np.einsum("bsii->b", R[..., 0] + 1j * R[..., 1])
        assert np.allclose(tr, np.round(tr.real[0]), atol=1e-8)
        E = f["/Measurements/Stage0/Energy/bins"]
        assert np.all(np.isfinite(E)) and np.all(E[:, 0] != 0.0)
