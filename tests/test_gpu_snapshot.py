"""The FP64 engine replays the reference's seeded snapshots through the C ABI.

The engine takes the reference's own random streams at its two injection points: the field
uniforms of every step (sfq_engine_propagate_host, the nwalk x nchol draw of assemble_X) and the
comb's uniform (sfq_engine_population_control_uniform).  Driven in run_afqmc's order it must
reproduce, step by step, the oracle's energy-estimator series, and through it the snapshot the
reference recorded, to the reference's own 1e-9: BH with an RHF trial and CLOSED walkers;
COLLINEAR walkers with BH's UHF and RHF trials and Li's polarized ROHF trial (no down electrons);
NONCOLLINEAR walkers with BH's RHF and UHF trials upgraded to spinors and a GHF trial; and the
34-determinant CASCI trials with each walker type.
"""
import numpy as np
import pytest

from oracle import afqmc_oracle as O
from oracle.mt19937 import HostRandomGenerator, split_seed
from safire_b200 import afqmc as A
from safire_b200 import capi, synthetic
from tests.golden_io import (SNAPSHOT_OBSERVABLES, bh_snapshot, engine_system, oracle_hamiltonian, snapshot,
                             snapshot_match)

pytestmark = pytest.mark.gpu

CASES = ["bh_rhf_closed", "bh_uhf_collinear", "bh_rhf_collinear", "li_rohf_collinear",
         "bh_rhf_noncollinear", "bh_uhf_noncollinear", "bh_ghf_noncollinear",
         # 34-determinant CASCI trials
         "bh_rcasci_rhf_closed", "bh_rcasci_rhf_collinear", "bh_rcasci_rhf_noncollinear",
         "bh_rcasci_uhf_collinear", "bh_rcasci_uhf_noncollinear", "bh_rcasci_ghf_noncollinear"]


def _system(snap):
    return engine_system(snap)


def _oracle_hamiltonian(snap):
    return oracle_hamiltonian(snap)


def _engine_series(snap, system=None):
    st = snap["settings"]
    eng = A.AfqmcEngine(system or _system(snap), st["nwalk"], dt=st["dt"], seed=0, precision=capi.PRECISION_FP64)
    walker_rng = HostRandomGenerator(split_seed(st["seed"], 0, 0))
    field_rng = HostRandomGenerator(split_seed(st["seed"], 0, 1))
    E_init = eng.init()
    _, series = eng.run_with_streams(st["steps"], E_init, field_rng.uniforms, lambda: walker_rng.uniforms(1)[0],
                                     ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                     equilibration_steps=st["equilibration_steps"],
                                     measure_interval=st["measure_interval"])
    rows = eng.walker_buffer()
    SM, _ = eng.walkers()
    eng.close()
    return E_init, series, rows, SM


@pytest.mark.parametrize("case", CASES)
def test_engine_reproduces_reference_snapshot(case):
    snap = snapshot(case)
    st = snap["settings"]
    Eshift, series, rows, SM = _engine_series(snap)
    E_init, _, oracle_series = O.run_seeded(_oracle_hamiltonian(snap), st["nwalk"], st["dt"], st["steps"],
                                            st["seed"], ortho_interval=st["ortho_interval"],
                                            pop_interval=st["pop_interval"], measure_interval=st["measure_interval"])
    assert abs(Eshift - E_init) < 1e-12 * abs(E_init)
    for k in SNAPSHOT_OBSERVABLES:
        a, b = np.asarray(series[k]), np.asarray(oracle_series[k])
        assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, float(np.max(np.abs(b)))), k
        assert snapshot_match(series[k], snap["recorded"][k], O.rebinned_average) is not None, k
    if st["walker_type"] == "COLLINEAR":
        # the reference's walker rows: the up block (M x nup), then the down block (M x ndn)
        nup = (snap["PsiT_up_dets"][0] if "ci_dets" in snap else snap["PsiT_up"]).shape[0]
        W, M, N = SM.shape
        assert np.array_equal(rows[:, :M * nup].reshape(W, M, nup), SM[:, :, :nup])
        assert np.array_equal(rows[:, M * nup:M * N].reshape(W, M, N - nup), SM[:, :, nup:])


def test_collinear_with_identical_spins_is_closed():
    """COLLINEAR walkers with the RHF orbitals for both spins follow the CLOSED walk on the GPU too."""
    snap = bh_snapshot()
    spec = synthetic.SystemSpec(M=snap["hcore"].shape[0], N=2 * snap["PsiT"].shape[0], Nc=snap["Likn"].shape[2],
                                decay=0.0)
    coll = synthetic.System(spec, snap["hcore"], snap["Likn"], np.concatenate([snap["PsiT"], snap["PsiT"]]),
                            snap["E0"], nel_dn=snap["PsiT"].shape[0])
    _, closed_series, _, _ = _engine_series(snap)
    _, coll_series, _, _ = _engine_series(snap, coll)
    for k in ("Energy", "ExchangeEnergy", "CoulombEnergy", "Overlap"):
        a, b = np.asarray(closed_series[k]), np.asarray(coll_series[k])
        assert np.max(np.abs(a - b)) < 1e-10 * np.max(np.abs(a)), k


def test_back_propagation_inside_device_blocks_matches_the_host_loop():
    """Blocks keep the back-propagation history on the device (field ring and weight-factor slots
    from a device-side position): anchored after 4 steps, 4 more steps with a comb inside, the
    back-propagated RDMs and observables equal the host loop's."""
    snap = bh_snapshot()
    sched = dict(ortho_interval=2, pop_interval=3, equilibration_steps=0, measure_interval=2)
    out = []
    for use_block in (False, True):
        eng = A.AfqmcEngine(_system(snap), 16, dt=0.01, seed=9, precision=capi.PRECISION_FP64)
        E = eng.init()
        eng.enable_back_propagation(4)
        for b in range(2):
            run = eng.run_block if use_block else eng.run
            E, _ = run(4, E, step0=4 * b, **sched)
            if b == 0:
                eng.bp_anchor()
        r = eng.measure_bp_rdms(4, ortho_interval=2)
        r.update(eng.measure_bp_observables(4, ortho_interval=2))
        out.append((r, eng.walkers()[0]))
        with pytest.raises(capi.SafireError) as ex:
            eng.measure_bp_rdms(5)  # longer than the ring
        assert ex.value.code == 2
        eng.close()
    (rh, Sh), (rd, Sd) = out
    assert np.max(np.abs(Sh - Sd)) <= 1e-12 * np.max(np.abs(Sh))
    assert rh.keys() == rd.keys() and len(rh) == 4
    for k in rh:
        assert np.max(np.abs(rh[k] - rd[k])) <= 1e-11 * max(1.0, float(np.max(np.abs(rh[k])))), k


@pytest.mark.parametrize("case", ["bh_uhf_collinear", "bh_ghf_noncollinear", "bh_rcasci_rhf_closed"])
def test_spin_walkers_rejected_in_mixed_precision(case):
    with pytest.raises(capi.SafireError) as ex:
        A.AfqmcEngine(_system(snapshot(case)), 8, dt=0.01, precision=capi.PRECISION_MIXED)
    assert ex.value.code == 3  # SFQ_ERR_UNSUPPORTED


def test_comb_uniform_rejected_outside_unit_interval():
    s = synthetic.make_system(synthetic.CFG_SMALL)
    eng = A.AfqmcEngine(s, 8, dt=0.005, seed=1, precision=capi.PRECISION_FP64)
    eng.init()
    for r in (-0.5, 1.0, float("nan")):
        with pytest.raises(capi.SafireError) as ex:
            eng.population_control(uniform=r)
        assert ex.value.code == 2
    eng.close()


RDM_CASES = ["bh_rhf_closed", "bh_uhf_collinear", "bh_uhf_noncollinear", "bh_rcasci_uhf_collinear",
             "bh_rcasci_uhf_noncollinear", "li_rohf_collinear"]


@pytest.mark.parametrize("case", RDM_CASES)
def test_engine_reproduces_recorded_rdms(case):
    """sfq_engine_measure_rdm every 2 steps and sfq_engine_measure_bp_rdm over 2 steps (with path
    restoration) in the replay: the mixed and back-propagated one-body and folded diagonal two-body
    RDMs against the oracle's per measurement and the recorded means / errors."""
    snap = snapshot(case)
    st = snap["settings"]
    eng = A.AfqmcEngine(_system(snap), st["nwalk"], dt=st["dt"], seed=0, precision=capi.PRECISION_FP64)
    walker_rng = HostRandomGenerator(split_seed(st["seed"], 0, 0))
    field_rng = HostRandomGenerator(split_seed(st["seed"], 0, 1))
    _, series = eng.run_with_streams(st["steps"], eng.init(), field_rng.uniforms, lambda: walker_rng.uniforms(1)[0],
                                     ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                     equilibration_steps=st["equilibration_steps"],
                                     measure_interval=st["measure_interval"], mixed_interval=snap["mixed_interval"],
                                     bp_steps=snap["bp_steps"], bp_ortho_interval=snap["bp_ortho_interval"])
    eng.close()
    _, _, oracle_series = O.run_seeded(_oracle_hamiltonian(snap), st["nwalk"], st["dt"], st["steps"], st["seed"],
                                       ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                       measure_interval=st["measure_interval"], mixed_interval=snap["mixed_interval"],
                                       bp_steps=snap["bp_steps"], bp_ortho_interval=snap["bp_ortho_interval"])
    rdms = [k for k in snap["recorded"] if k.startswith(("MixedEstimator", "BackPropEstimator"))]
    assert len(rdms) == 4
    for k in rdms:
        a, b = np.asarray(series[k]), np.asarray(oracle_series[k])
        assert a.shape == b.shape
        assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, float(np.max(np.abs(b)))), k
        assert snapshot_match(series[k], snap["recorded"][k], O.rebinned_average) is not None, k
