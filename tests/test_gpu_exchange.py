"""The sharded walker exchange on the device (sfq_engine_pack_walkers / unpack_walkers /
copy_walkers, driven by safire_b200.popcontrol.engine_population_control).

* One rank: engine_population_control on an engine equals the engine's own single-rank comb
  (engine.population_control with the same uniform) bit for bit -- walkers, properties and the
  next step's energies.
* Two ranks on one GPU: two engines hold the two ranks' shares; the plan of the global comb is
  carried out with the engines' row calls, the rows handed from the sending engine's buffer to the
  receiving one in plan order (what NCCL send/recv does between GPUs), and each engine ends with
  exactly the walker table the same moves give on the host.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from safire_b200 import afqmc as A  # noqa: E402
from safire_b200 import capi, synthetic  # noqa: E402
from safire_b200 import popcontrol as P  # noqa: E402


def _engine(s, W, seed, steps=3):
    e = A.AfqmcEngine(s, W, dt=0.005, seed=seed)
    Esh = e.init()
    for st in range(steps):
        e.propagate(Esh, st)
    return e


def test_one_rank_equals_the_engine_comb():
    s = synthetic.make_system(synthetic.CFG_SMALL)
    a, b = _engine(s, 48, 11), _engine(s, 48, 11)
    r = 0.3719
    a.population_control(uniform=r)
    P.engine_population_control(None, b, r)
    Sa, pa = a.walkers()
    Sb, pb = b.walkers()
    assert np.array_equal(Sa, Sb)
    for k in capi.PROPS:
        assert np.array_equal(pa[k], pb[k]), k
    Ea, Eb = a.energy(), b.energy()
    assert np.max(np.abs(Ea - Eb)) <= 1e-12 * np.max(np.abs(Ea))
    a.propagate(0.0, 10)
    b.propagate(0.0, 10)
    assert np.array_equal(a.walkers()[0], b.walkers()[0])
    a.close()
    b.close()


def _host_moves(tables, offspring, counts):
    """The same plan applied to host copies of the tables (the expected result)."""
    out = [(S.copy(), pr.copy()) for S, pr in tables]
    queues = {}
    for rank, (S, pr) in enumerate(tables):
        sends, _, _ = P.local_moves(offspring, counts, rank)
        for walker, dst in sends:
            queues.setdefault((rank, dst), []).append((S[walker].copy(), pr[:, walker].copy()))
    for rank in range(len(tables)):
        S, pr = out[rank]
        _, recvs, copies = P.local_moves(offspring, counts, rank)
        for slot, src in recvs:
            S[slot], pr[:, slot] = queues[(src, rank)].pop(0)
        pr[0] = pr[0] / np.abs(pr[0])
        for src, dst in copies:
            S[dst] = S[src]
            pr[:, dst] = pr[:, src]
    return out


@pytest.mark.parametrize("counts,boost", [((24, 40), 3.0), ((40, 24), 0.2), ((32, 32), 1.0)])
def test_two_ranks_on_device_rows(counts, boost):
    s = synthetic.make_system(synthetic.CFG_SMALL)
    engines = [_engine(s, n, 100 + i) for i, n in enumerate(counts)]
    # tilt the weights so that walkers have to move between the ranks
    SM0, p0 = engines[0].walkers()
    p0["WEIGHT"] = p0["WEIGHT"] * boost
    engines[0].set_walkers(None, p0)
    tables = []
    for e in engines:
        S, pr = e.walkers()
        tables.append((S, np.stack([pr[k] for k in capi.PROPS])))
    w = np.concatenate([np.abs(t[1][0]) for t in tables])
    offspring = P.comb(w, 0.61, w.size)
    expect = _host_moves(tables, offspring, list(counts))

    width = 2 * engines[0].walker_row_elems()
    assert width == 2 * (s.M * s.N + 8)
    queues = {}
    moves = [P.local_moves(offspring, list(counts), r) for r in range(len(counts))]
    nmoved = 0
    for rank, e in enumerate(engines):
        sends = moves[rank][0]
        if sends:
            rows = torch.empty((len(sends), width), dtype=torch.float64, device=e.exchange_device)
            e.pack_walkers([wk for wk, _ in sends], rows)
            for i, (_, dst) in enumerate(sends):
                queues.setdefault((rank, dst), []).append(rows[i])
            nmoved += len(sends)
    assert nmoved > 0 or boost == 1.0
    for rank, e in enumerate(engines):
        _, recvs, copies = moves[rank]
        if recvs:
            rows = torch.stack([queues[(src, rank)].pop(0) for _, src in recvs]).contiguous()
            torch.cuda.synchronize()
            e.unpack_walkers([slot for slot, _ in recvs], rows)
        e.copy_walkers(copies, normalize=True)
    for rank, e in enumerate(engines):
        S, pr = e.walkers()
        assert S.shape[0] == counts[rank]
        assert np.array_equal(S, expect[rank][0])
        got = np.stack([pr[k] for k in capi.PROPS])
        assert np.array_equal(got[1:], expect[rank][1][1:])
        # w / |w|: the device's hypot and the host's may differ in the last bit
        assert np.max(np.abs(got[0] - expect[rank][1][0])) <= 4e-16
        e.close()


def test_row_calls_reject_bad_slots_and_pairs():
    s = synthetic.make_system(synthetic.CFG_SMALL)
    e = _engine(s, 8, 3, steps=0)
    rows = torch.empty((1, 2 * e.walker_row_elems()), dtype=torch.float64, device=e.exchange_device)
    with pytest.raises(capi.SafireError):
        e.pack_walkers([8], rows)             # slot outside [0, 8)
    with pytest.raises(capi.SafireError):
        e.copy_walkers([(0, 1), (1, 2)])      # a destination that is also a source
    with pytest.raises(capi.SafireError):
        e.copy_walkers([(0, 1), (2, 1)])      # the same destination twice
    e.enable_back_propagation(4)
    with pytest.raises(capi.SafireError) as ei:
        e.pack_walkers([0], rows)             # the rows carry no back-propagation history
    assert ei.value.code == 3
    e.close()
