"""The FP64 engine replays the reference's seeded BH snapshot through the C ABI.

The engine takes the reference's own random streams at its two injection points: the field
uniforms of every step (sfq_engine_propagate_host, the nwalk x nchol draw of assemble_X) and the
comb's uniform (sfq_engine_population_control_uniform).  Driven in run_afqmc's order it must
reproduce, step by step, the oracle's energy-estimator series, and through it the snapshot the
reference recorded, to the reference's own 1e-9.
"""
import numpy as np
import pytest

from oracle import afqmc_oracle as O
from oracle.mt19937 import HostRandomGenerator, split_seed
from safire_b200 import afqmc as A
from safire_b200 import capi, synthetic
from tests.golden_io import SNAPSHOT_OBSERVABLES, bh_snapshot, snapshot_match

pytestmark = pytest.mark.gpu


def _engine_series(snap):
    st = snap["settings"]
    M, N = snap["PsiT"].shape[1], snap["PsiT"].shape[0]
    Nc = snap["Likn"].shape[2]
    system = synthetic.System(synthetic.SystemSpec(M=M, N=N, Nc=Nc, decay=0.0), snap["hcore"], snap["Likn"],
                              snap["PsiT"], snap["E0"])
    eng = A.AfqmcEngine(system, st["nwalk"], dt=st["dt"], seed=0, precision=capi.PRECISION_FP64)
    walker_rng = HostRandomGenerator(split_seed(st["seed"], 0, 0))
    field_rng = HostRandomGenerator(split_seed(st["seed"], 0, 1))
    E_init = eng.init()
    _, series = eng.run_with_streams(st["steps"], E_init, field_rng.uniforms, lambda: walker_rng.uniforms(1)[0],
                                     ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                     equilibration_steps=st["equilibration_steps"],
                                     measure_interval=st["measure_interval"])
    eng.close()
    return E_init, series


def test_engine_reproduces_reference_snapshot():
    snap = bh_snapshot()
    st = snap["settings"]
    Eshift, series = _engine_series(snap)
    ham = O.Hamiltonian(snap["hcore"], snap["Likn"], snap["PsiT"], snap["E0"])
    E_init, _, oracle_series = O.run_seeded(ham, st["nwalk"], st["dt"], st["steps"], st["seed"],
                                            ortho_interval=st["ortho_interval"], pop_interval=st["pop_interval"],
                                            measure_interval=st["measure_interval"])
    assert abs(Eshift - E_init) < 1e-12 * abs(E_init)
    for k in SNAPSHOT_OBSERVABLES:
        a, b = np.asarray(series[k]), np.asarray(oracle_series[k])
        assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, float(np.max(np.abs(b)))), k
        assert snapshot_match(series[k], snap["recorded"][k], O.rebinned_average) is not None, k


def test_comb_uniform_rejected_outside_unit_interval():
    s = synthetic.make_system(synthetic.CFG_SMALL)
    eng = A.AfqmcEngine(s, 8, dt=0.005, seed=1, precision=capi.PRECISION_FP64)
    eng.init()
    for r in (-0.5, 1.0, float("nan")):
        with pytest.raises(capi.SafireError) as ex:
            eng.population_control(uniform=r)
        assert ex.value.code == 2
    eng.close()
