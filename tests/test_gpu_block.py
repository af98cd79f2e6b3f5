"""The device-resident block driver (sfq_engine_block*): the same run_afqmc loop as sfq_engine_run,
with Eshift, the step counter and the measurements on the device and each block replayed from a
CUDA graph, gives the host loop's results."""
import time

import numpy as np
import pytest

from safire_b200 import afqmc as A
from safire_b200 import capi, synthetic

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _pair(prec=capi.PRECISION_FP64, spec=synthetic.CFG_SMALL, W=32, seed=5):
    s = synthetic.make_system(spec)
    e1 = A.AfqmcEngine(s, W, dt=0.005, seed=seed, precision=prec)
    e2 = A.AfqmcEngine(s, W, dt=0.005, seed=seed, precision=prec)
    return e1, e2


SCHED = dict(ortho_interval=5, pop_interval=20, equilibration_steps=20, measure_interval=10)


def test_block_matches_host_loop():
    host, dev = _pair()
    E0 = host.init()
    dev.init()
    Eh, mh = host.run(40, E0, **SCHED)
    Ed, md = dev.run_block(40, E0, **SCHED)
    assert len(md) == len(mh) == 2
    assert abs(Ed - Eh) < 1e-10 * abs(Eh)  # Eshift relaxed on the device during equilibration
    assert _rel(md, mh) < 1e-9
    S1, p1 = host.walkers()
    S2, p2 = dev.walkers()
    assert _rel(S2, S1) < 1e-9
    assert _rel(p2["WEIGHT"], p1["WEIGHT"]) < 1e-9
    host.close()
    dev.close()


def test_consecutive_blocks_and_graph_replay():
    host, dev = _pair(seed=9)
    E0 = host.init()
    dev.init()
    Eh, mh = host.run(60, E0, **SCHED)
    E1, m1 = dev.run_block(20, E0, step0=0, **SCHED)   # equilibration schedule
    E2, m2 = dev.run_block(20, E1, step0=20, **SCHED)  # measurement schedule (captured)
    E3, m3 = dev.run_block(20, E2, step0=40, **SCHED)  # the same schedule: replayed graph
    md = np.concatenate([m1, m2, m3])
    assert abs(E3 - Eh) < 1e-10 * abs(Eh)
    assert _rel(md, mh) < 1e-9
    S1, _ = host.walkers()
    S2, _ = dev.walkers()
    assert _rel(S2, S1) < 1e-9
    host.close()
    dev.close()


def test_block_async_query_result():
    a, b = _pair(seed=3)
    E0 = a.init()
    b.init()
    Ea, ma = a.run_block(20, E0, equilibration_steps=0, measure_interval=20, ortho_interval=5, pop_interval=20)
    b.block_async(20, E0, equilibration_steps=0, measure_interval=20, ortho_interval=5, pop_interval=20)
    t0 = time.time()
    while not b.block_query():
        assert time.time() - t0 < 60
        time.sleep(0.001)
    Eb, mb = b.block_result()
    assert Eb == Ea
    assert np.array_equal(ma, mb)
    a.close()
    b.close()


@pytest.mark.parametrize("prec", [capi.PRECISION_MIXED, capi.PRECISION_INT8X3])
def test_mixed_block_matches_host_loop(prec):
    host, dev = _pair(prec=prec, spec=synthetic.CFG_MEDIUM, W=16, seed=2)
    E0 = host.init()
    dev.init()
    sched = dict(ortho_interval=5, pop_interval=20, equilibration_steps=0, measure_interval=10)
    Eh, mh = host.run(20, E0, **sched)
    Ed, md = dev.run_block(20, E0, **sched)
    assert Ed == Eh  # no relaxation: Eshift is the given one throughout
    assert _rel(md, mh) < 1e-12  # the same kernels on the same data, launched from a graph
    S1, _ = host.walkers()
    S2, _ = dev.walkers()
    assert _rel(S2, S1) < 1e-12
    host.close()
    dev.close()


def test_steered_block_matches_host_loop():
    """steer_eshift: Eshift keeps relaxing after equilibration, measurements continue."""
    host, dev = _pair(seed=13)
    E0 = host.init()
    dev.init()
    sched = dict(ortho_interval=5, pop_interval=20, equilibration_steps=10, measure_interval=10, relax=0.1,
                 steer=True)
    Eh, mh = host.run(40, E0, **sched)
    Ed, md = dev.run_block(40, E0, **sched)
    assert len(md) == len(mh) == 3
    assert abs(Ed - Eh) < 1e-10 * abs(Eh)
    assert _rel(md, mh) < 1e-9
    host.close()
    dev.close()
