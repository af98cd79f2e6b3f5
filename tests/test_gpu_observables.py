"""TwoRDM, SpinCorr and PairCorr of the mixed and back-propagated estimators on the B200
(sfq_engine_measure_observables / sfq_engine_measure_bp_observables) against the oracle's
restatement of Observables/twordm.hpp, spincorr.hpp and paircorr.hpp, measured along the replay of
the reference's seeded BH runs (the same schedule as the recorded one- and two-body RDMs): CLOSED,
COLLINEAR and NONCOLLINEAR walkers, each observable where the reference measures it; and the
time-evolved back-propagation estimator (sfq_engine_te_*) against the oracle's restatement."""
import numpy as np
import pytest

from oracle import afqmc_oracle as O
from oracle.mt19937 import HostRandomGenerator, split_seed
from safire_b200 import afqmc as A
from safire_b200 import capi
from tests.golden_io import engine_system, oracle_hamiltonian, snapshot

pytestmark = pytest.mark.gpu


def _maps(M):
    return np.array([[(i + 1) % M if i % 3 != 2 else -1 for i in range(M)], [M - 1 - i for i in range(M)]])


CASES = [("bh_rhf_closed", True, True, False), ("bh_uhf_collinear", True, True, True),
         ("bh_uhf_noncollinear", False, True, True)]


@pytest.mark.parametrize("case,two,spin,pair", CASES)
def test_observables_match_the_oracle_along_the_seeded_replay(case, two, spin, pair):
    snap = snapshot(case)
    st = snap["settings"]
    M = snap["hcore"].shape[0]
    obs = dict(two_rdm=two, spin_corr=spin, pair_maps=_maps(M) if pair else None)
    eng = A.AfqmcEngine(engine_system(snap), st["nwalk"], dt=st["dt"], seed=0, precision=capi.PRECISION_FP64)
    walker_rng = HostRandomGenerator(split_seed(st["seed"], 0, 0))
    field_rng = HostRandomGenerator(split_seed(st["seed"], 0, 1))
    _, series = eng.run_with_streams(st["steps"], eng.init(), field_rng.uniforms, lambda: walker_rng.uniforms(1)[0],
                                     ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                     equilibration_steps=st["equilibration_steps"],
                                     measure_interval=st["measure_interval"], mixed_interval=snap["mixed_interval"],
                                     bp_steps=snap["bp_steps"], bp_ortho_interval=snap["bp_ortho_interval"],
                                     observables=obs)
    eng.close()
    _, _, oracle = O.run_seeded(oracle_hamiltonian(snap), st["nwalk"], st["dt"], st["steps"], st["seed"],
                                ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                measure_interval=st["measure_interval"], mixed_interval=snap["mixed_interval"],
                                bp_steps=snap["bp_steps"], bp_ortho_interval=snap["bp_ortho_interval"],
                                observables=obs)
    names = [k for k in series if k.endswith(("TwoRDM", "SpinCorr", "PairCorr")) and "Diagonal" not in k]
    expect = (2 if two else 0) + (2 if spin else 0) + (2 if pair else 0)  # mixed and back-propagated
    assert len(names) == expect, names
    for k in names:
        a, b = np.asarray(series[k]), np.asarray(oracle[k])
        assert a.shape == b.shape, k
        assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, float(np.max(np.abs(b)))), k


@pytest.mark.parametrize("case,two,pair", [("bh_rcasci_rhf_closed", True, False), ("bh_rcasci_uhf_collinear", True, True),
                                           ("bh_rcasci_ghf_noncollinear", False, True)])
def test_multi_determinant_observables_match_the_oracle(case, two, pair):
    """The reference's 34-determinant BH CASCI trials: TwoRDM, SpinCorr and PairCorr of the mixed and
    back-propagated estimators summed over the references (each determinant's G with its
    coefficient, the referenceLoop of twordm.hpp / spincorr.hpp / paircorr.hpp), along 8 steps of
    the seeded replay, against the oracle's restatement."""
    snap = snapshot(case)
    st = snap["settings"]
    M = snap["hcore"].shape[0]
    steps = 8
    obs = dict(two_rdm=two, spin_corr=True, pair_maps=_maps(M) if pair else None)
    kw = dict(ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"], measure_interval=st["measure_interval"],
              mixed_interval=snap.get("mixed_interval") or 2, bp_steps=snap.get("bp_steps") or [2],
              bp_ortho_interval=snap.get("bp_ortho_interval") or 10)
    eng = A.AfqmcEngine(engine_system(snap), st["nwalk"], dt=st["dt"], seed=0, precision=capi.PRECISION_FP64)
    walker_rng = HostRandomGenerator(split_seed(st["seed"], 0, 0))
    field_rng = HostRandomGenerator(split_seed(st["seed"], 0, 1))
    _, series = eng.run_with_streams(steps, eng.init(), field_rng.uniforms, lambda: walker_rng.uniforms(1)[0],
                                     equilibration_steps=st["equilibration_steps"], observables=obs, **kw)
    eng.close()
    _, _, oracle = O.run_seeded(oracle_hamiltonian(snap), st["nwalk"], st["dt"], steps, st["seed"], observables=obs,
                                equilibration_steps=st["equilibration_steps"], **kw)
    names = [k for k in series if k.endswith(("TwoRDM", "SpinCorr", "PairCorr")) and "Diagonal" not in k]
    assert len(names) == (2 if two else 0) + 2 + (2 if pair else 0), names
    for k in names:
        a, b = np.asarray(series[k]), np.asarray(oracle[k])
        assert a.shape == b.shape and len(a) > 0, k
        assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, float(np.max(np.abs(b)))), k


def test_observables_refused_where_the_reference_refuses_them():
    closed = engine_system(snapshot("bh_rhf_closed"))
    nonc = engine_system(snapshot("bh_uhf_noncollinear"))
    e = A.AfqmcEngine(closed, 8, dt=0.01, seed=1, precision=capi.PRECISION_FP64)
    e.init()
    with pytest.raises(capi.SafireError) as ex:
        e.measure_observables(two_rdm=False, spin_corr=False, pair_maps=_maps(closed.M))  # paircorr.hpp:37-40
    assert ex.value.code == 3
    e.close()
    e = A.AfqmcEngine(nonc, 8, dt=0.01, seed=1, precision=capi.PRECISION_FP64)
    e.init()
    with pytest.raises(capi.SafireError) as ex:
        e.measure_observables(two_rdm=True, spin_corr=False)  # twordm.hpp:34-36
    assert ex.value.code == 3
    e.close()
    e = A.AfqmcEngine(closed, 8, dt=0.01, seed=1, precision=capi.PRECISION_INT8X3)
    e.init()
    with pytest.raises(capi.SafireError) as ex:
        e.measure_observables(two_rdm=True, spin_corr=True)  # the estimators are FP64
    assert ex.value.code == 3
    e.close()


@pytest.mark.parametrize("case,extra", [("bh_rhf_closed", False), ("bh_uhf_collinear", True),
                                        ("bh_uhf_noncollinear", False), ("bh_rcasci_rhf_closed", False),
                                        ("bh_rcasci_uhf_collinear", False), ("bh_rcasci_ghf_noncollinear", False)])
def test_time_evolved_back_propagation_matches_the_oracle(case, extra):
    """TimeEvolvedBPEstimator over lengths 2 and 4 (two segments per window, combs and
    orthogonalizations inside it) along the seeded BH replay: the one-body and diagonal two-body
    RDMs and the other observables of the dressed Green's functions, against the oracle's
    restatement (with extra path restoration for the collinear case); the CASCI trials dress every
    reference's G and weight it by its coefficient (CLOSED overlaps doubled)."""
    snap = snapshot(case)
    st = snap["settings"]
    M = snap["hcore"].shape[0]
    nonc = st["walker_type"] == "NONCOLLINEAR"
    obs = dict(two_rdm=not nonc, spin_corr=True, pair_maps=_maps(M) if st["walker_type"] != "CLOSED" else None)
    kw = dict(ortho_interval=st["ortho_interval"], pop_interval=3, measure_interval=st["measure_interval"])
    eng = A.AfqmcEngine(engine_system(snap), st["nwalk"], dt=st["dt"], seed=0, precision=capi.PRECISION_FP64)
    walker_rng = HostRandomGenerator(split_seed(st["seed"], 0, 0))
    field_rng = HostRandomGenerator(split_seed(st["seed"], 0, 1))
    _, series = eng.run_with_streams(12, eng.init(), field_rng.uniforms, lambda: walker_rng.uniforms(1)[0],
                                     equilibration_steps=0, te_steps=[2, 4], te_extra_path_restoration=extra,
                                     observables=obs, **kw)
    eng.close()
    _, _, oracle = O.run_seeded(oracle_hamiltonian(snap), st["nwalk"], st["dt"], 12, st["seed"], te_steps=[2, 4],
                                te_extra_path_restoration=extra, observables=obs, **kw)
    names = [k for k in series if k.startswith("TimeEvolvedBP/")]
    assert len(names) == 2 * (2 + sum(1 for v in (obs["two_rdm"], obs["spin_corr"], obs["pair_maps"] is not None) if v))
    for k in names:
        a, b = np.asarray(series[k]), np.asarray(oracle[k])
        assert a.shape == b.shape and len(a) == 3, k  # lengths 2 and 4 of windows at steps 1, 5, 9
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, float(np.max(np.abs(b)))), k
