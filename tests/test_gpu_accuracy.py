"""Block energy of the INT8X3 engine against the FP64 drop-in at the headline size (M=400, N=100+100,
Nchol=2400, 256 walkers, dt = 0.0005), run_afqmc's equilibration schedule (orthogonalization every 5
steps, comb every 20, Eshift relaxed every step), 25 steps, seeded fields identical in both runs.

* Measurement: the energy of identical walkers differs by far less than 0.1 mHa (the exchange tensor
  comes from exact int32 products).  The split-BF16 engine, whose tensor-core FP32 accumulation
  rounds toward zero, is off by tens of mHa on the same walkers: that bias is what the int8 slices
  remove.
* Trajectories: the fixed-point slices (2^-24 of each row's largest entry) leave unbiased noise of
  a few 1e-7 per step in the propagated walkers, so one seeded 25-step block moves by about
  0.1 mHa either way; over several seeds the mean difference is within 0.1 mHa of zero.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from safire_b200 import afqmc, capi, synthetic  # noqa: E402

W = 256
DT = 0.0005
STEPS = 25
RELAX = 1.0 - math.exp(-10.0 / 100)
SEEDS = (1000, 1, 2, 3, 4, 5)


@pytest.fixture(scope="module")
def system():
    return synthetic.make_system(synthetic.CFG_LARGE)


def _block_energy(s, prec, seed):
    eng = afqmc.AfqmcEngine(s, W, dt=DT, seed=seed, precision=prec)
    Esh = eng.init()
    for st in range(STEPS):
        eng.propagate(Esh, st)
        if st % 5 == 0:
            eng.orthogonalize()
        if st % 20 == 0:
            eng.population_control(st)
        Esh += RELAX * (eng.averages()[0] - Esh)
    E = eng.measure()["Energy"].real
    return eng, E


def test_int8x3_measures_identical_walkers_without_bias(system):
    e64, _ = _block_energy(system, capi.PRECISION_FP64, 1000)
    SM, pr = e64.walkers()
    E64 = e64.measure()["Energy"].real
    e64.close()
    out = {}
    for prec in (capi.PRECISION_INT8X3, capi.PRECISION_MIXED):
        eng = afqmc.AfqmcEngine(system, W, dt=DT, seed=1000, precision=prec)
        eng.set_walkers(SM, pr)
        out[prec] = 1e3 * (eng.measure()["Energy"].real - E64)
        eng.close()
    assert abs(out[capi.PRECISION_INT8X3]) < 0.01, out
    assert abs(out[capi.PRECISION_MIXED]) > 1.0, out  # the round-toward-zero bias of split-BF16


def test_int8x3_block_energy_within_0p1_mha_of_fp64(system):
    deltas = []
    for seed in SEEDS:
        e64, E64 = _block_energy(system, capi.PRECISION_FP64, seed)
        e64.close()
        e8, E8 = _block_energy(system, capi.PRECISION_INT8X3, seed)
        e8.close()
        deltas.append(1e3 * (E8 - E64))
    d = np.array(deltas)
    sem = d.std(ddof=1) / math.sqrt(len(d))
    print("block energy INT8X3 - FP64 (mHa) per seed:", np.round(d, 4), "mean", d.mean(), "+-", sem)
    assert abs(d.mean()) < 0.1, d
    assert abs(d.mean()) < 3 * sem + 0.02, d   # no bias beyond the seeds' spread
    assert np.max(np.abs(d)) < 0.3, d
