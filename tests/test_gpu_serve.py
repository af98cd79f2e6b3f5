"""Serving loop on the GPU: each result is the same alone and in the mix; eviction keeps walkers."""
import numpy as np
import pytest

from safire_b200 import afqmc as A
from safire_b200 import capi, synthetic
from safire_b200.serve import Server

pytestmark = pytest.mark.gpu

BLK = dict(steps=10, ortho_interval=5, pop_interval=20, equilibration_steps=0, measure_interval=10)


def _systems():
    return [synthetic.make_system(synthetic.SystemSpec(M=M, N=M // 4, Nc=6 * M, decay=float(M), seed=40 + i))
            for i, M in enumerate((48, 64, 32))]


def _add_all(srv, systems):
    return [srv.add_system(s, 16, dt=0.002, seed=500 + i, precision=capi.PRECISION_MIXED)
            for i, s in enumerate(systems)]


def test_same_alone_and_in_the_mix():
    systems = _systems()
    alone = Server(hbm_budget_gb=20.0, max_inflight=4)
    ids = _add_all(alone, systems)
    res_alone = []
    for _ in range(3):
        r = alone.submit(ids[0], **BLK)
        alone.drain([r])
        res_alone.append(alone.request(r))
    alone.close()
    mix = Server(hbm_budget_gb=20.0, max_inflight=4)
    ids = _add_all(mix, systems)
    res_mix = []
    for _ in range(3):
        rs = [mix.submit(sid, **BLK) for sid in (ids[1], ids[0], ids[2])]  # overlapping on the GPU
        mix.drain(rs)
        res_mix.append(mix.request(rs[1]))
        assert all(mix.request(r)["status"] == 0 for r in rs)
    mix.close()
    for a, b in zip(res_alone, res_mix):
        assert a["status"] == b["status"] == 0
        assert a["step0"] == b["step0"]
        assert a["Eshift"] == b["Eshift"]
        assert np.array_equal(a["meas"], b["meas"])  # bit for bit: the systems share nothing


def test_server_matches_engine_blocks():
    s = _systems()[0]
    srv = Server(hbm_budget_gb=20.0, max_inflight=2)
    sid = srv.add_system(s, 16, dt=0.002, seed=500, precision=capi.PRECISION_MIXED)
    eng = A.AfqmcEngine(s, 16, dt=0.002, seed=500, precision=capi.PRECISION_MIXED)
    E = eng.init()
    for blk in range(2):
        r = srv.submit(sid, **BLK)
        srv.drain([r])
        got = srv.request(r)
        kw = {k: v for k, v in BLK.items() if k != "steps"}
        E, meas = eng.run_block(BLK["steps"], E, step0=10 * blk, **kw)
        assert got["Eshift"] == E
        assert np.array_equal(got["meas"], meas)
    eng.close()
    srv.close()


def test_eviction_restores_walkers():
    systems = _systems()[:2]
    big = Server(hbm_budget_gb=20.0, max_inflight=1)
    ids = _add_all(big, systems)
    ref = []
    for _ in range(2):
        for sid in ids:
            r = big.submit(sid, **BLK)
            big.drain([r])
            ref.append(big.request(r))
    big.close()
    # find a budget that holds one of the two engines but not both
    probe = Server(hbm_budget_gb=20.0, max_inflight=1)
    pid = _add_all(probe, systems)
    probe.warm(pid[0])
    b0 = probe.stats()["used_bytes"]
    probe.warm(pid[1])
    b1 = probe.stats()["used_bytes"] - b0
    probe.close()
    tight = Server(hbm_budget_gb=(max(b0, b1) * 1.05) / 1e9, max_inflight=1)
    ids = _add_all(tight, systems)
    got = []
    for _ in range(2):
        for sid in ids:
            r = tight.submit(sid, **BLK)
            tight.drain([r])
            got.append(tight.request(r))
            assert tight.stats()["resident"] == 1  # the other system was evicted
    tight.close()
    for a, b in zip(ref, got):
        assert a["Eshift"] == b["Eshift"]
        assert np.array_equal(a["meas"], b["meas"])
