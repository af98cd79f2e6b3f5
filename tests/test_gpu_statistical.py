"""The FP64 engine's own runs agree with the reference's statistical references.

The reference's long runs of BH (RHF trial, CLOSED walkers) and Li (polarized ROHF trial, COLLINEAR
walkers) -- dense Cholesky, 96 ranks x 16 walkers, 48000 steps of 0.01, 3000 of them equilibration
with a relaxing Eshift, population control, orthogonalization and a measurement every 10 steps --
recorded the mean and error of each energy.  The engine runs the same schedule on one GPU for the same
1536 walkers, with its own Philox fields and comb, as device-resident blocks; its means must agree
with the recorded ones under the reference's own statistical comparison -- in FP64, and with the
int8-slice products (INT8X3) on both fixtures.
"""
import numpy as np
import pytest

from oracle import afqmc_oracle as O
from safire_b200 import afqmc as A
from safire_b200 import capi
from tests.golden_io import bh_statistical, engine_system, snapshot, statistically_equal

pytestmark = pytest.mark.gpu

KEYS = ("Energy", "OnebodyEnergy", "ExchangeEnergy", "CoulombEnergy")


@pytest.mark.parametrize("prec", [capi.PRECISION_FP64, capi.PRECISION_INT8X3], ids=["fp64", "int8x3"])
@pytest.mark.parametrize("case", ["bh_rhf_closed", "li_rohf_collinear"])
def test_engine_agrees_with_reference_statistics(case, prec):
    snap, stat = snapshot(case), bh_statistical(case)
    assert snap["settings"]["walker_type"] == stat["walker_type"]
    eng = A.AfqmcEngine(engine_system(snap), stat["nwalk"], dt=stat["dt"], seed=2024, precision=prec)
    Eshift = eng.init()
    block = 50 * stat["measure_interval"]  # 50 measurements per device-resident block
    assert stat["steps"] % block == 0
    rows = []
    for b in range(stat["steps"] // block):
        Eshift, meas = eng.run_block(block, Eshift, ortho_interval=stat["ortho_interval"],
                                     pop_interval=stat["pop_interval"],
                                     equilibration_steps=stat["equilibration_steps"],
                                     measure_interval=stat["measure_interval"], relax=0.0, step0=b * block)
        rows.append(meas)
    eng.close()
    meas = np.concatenate(rows)
    n_expected = (stat["steps"] - stat["equilibration_steps"]) // stat["measure_interval"]
    assert meas.shape[0] == n_expected
    for i, k in enumerate(KEYS):
        series = meas[:, 2 * i] + 1j * meas[:, 2 * i + 1]
        mean, err = O.rebinned_average(series, 50)  # bins of 500 steps, longer than the correlation time
        ok, d, tol = statistically_equal(mean, err, *stat["recorded"][k])
        rm, re_ = stat["recorded"][k]
        print(f"{case} {prec} {k}: {mean.real:.6f} +- {abs(err):.6f} vs recorded {rm.real:.6f} +- {abs(re_):.6f}, "
              f"|d| = {d:.2e} <= {tol:.2e}")
        assert ok, (k, mean, err, stat["recorded"][k], d, tol)
