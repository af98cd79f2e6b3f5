"""Population control over walkers sharded across ranks (safire_b200.popcontrol): the native host
comb, exchange plan and per-rank moves (sfq_comb_host, sfq_plan_walker_exchange, sfq_walker_moves)
against the oracle's restatement, one rank against the oracle's single-rank comb, and two gloo ranks
on the CPU against one rank holding the whole population."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import afqmc_oracle as O
from safire_b200 import capi
from safire_b200 import popcontrol as P


@pytest.fixture(scope="module", autouse=True)
def built():
    from safire_b200 import build
    build.build()


def _table(nw, seed, rows=5, cols=2):
    rng = np.random.default_rng(seed)
    SM = rng.standard_normal((nw, rows, cols)) + 1j * rng.standard_normal((nw, rows, cols))
    props = rng.standard_normal((8, nw)) + 1j * rng.standard_normal((8, nw))
    w = np.exp(rng.standard_normal(nw))
    w[rng.integers(0, nw)] = 0.0            # a dead walker
    w[rng.integers(0, nw)] *= 12.0          # a heavy one
    props[P.WEIGHT] = w * np.exp(1j * rng.uniform(-0.3, 0.3, nw))
    return SM, props


def test_comb_matches_the_oracle():
    rng = np.random.default_rng(1)
    for n in (1, 2, 37, 500):
        for _ in range(20):
            w = np.abs(rng.standard_normal(n)) ** 3
            w[rng.random(n) < 0.2] = 0.0
            if not w.sum() > 1e-6:
                w[-1] = 1.0
            r = rng.uniform()
            for target in (n, max(1, n // 2), 2 * n):
                assert np.array_equal(P.comb(w, r, target), O.comb(w, r, target))


def test_comb_trailing_dead_walkers_and_collapse():
    """Teeth past the last live walker land on it (the iw == last clause), and a collapsed total
    weight is an error, not a division by zero."""
    w = np.array([0.5, 2.0, 0.0, 0.0])
    assert np.array_equal(P.comb(w, 0.999999, 4), O.comb(w, 0.999999, 4))
    assert P.comb(w, 0.999999, 4)[2:].sum() == 0
    with pytest.raises(capi.SafireError, match="WEIGHT_COLLAPSE"):
        P.comb(np.full(5, 1e-8), 0.5, 5)
    with pytest.raises(capi.SafireError, match="ARG"):
        P.comb(w, 1.0, 4)


def test_plan_and_moves_match_the_oracle():
    rng = np.random.default_rng(11)
    for _ in range(200):
        nranks = int(rng.integers(1, 7))
        counts = [int(c) for c in rng.integers(0, 9, nranks)]
        if sum(counts) == 0:
            counts[0] = 3
        ntot = sum(counts)
        w = np.abs(rng.standard_normal(ntot)) ** int(rng.integers(1, 5))
        off = O.comb(w, rng.uniform(), ntot)
        assert P.plan_walker_exchange(off, counts) == O.plan_walker_exchange(off, counts)
        for r in range(nranks):
            assert P.local_moves(off, counts, r) == O.walker_moves(off, counts, r)


def test_plan_rejects_a_population_that_changes():
    with pytest.raises(capi.SafireError, match="ARG"):
        P.plan_walker_exchange([2, 2, 1], [2, 2])       # 3 entries for 4 walkers
    with pytest.raises(capi.SafireError, match="ARG"):
        P.plan_walker_exchange([2, 0, 0, 1], [2, 2])    # 3 copies of 4 walkers
    with pytest.raises(capi.SafireError, match="ARG"):
        P.local_moves([1, 1, 1, 1], [2, 2], 2)          # no rank 2


@pytest.mark.parametrize("counts", [[6, 6], [5, 7, 4], [1, 9], [8, 0, 8]])
def test_plan_moves_excess_to_deficits(counts):
    rng = np.random.default_rng(sum(counts))
    for _ in range(30):
        ntot = sum(counts)
        off = P.comb(np.abs(rng.standard_normal(ntot)) ** 2, rng.uniform(), ntot)
        plan = P.plan_walker_exchange(off, counts)
        first = np.cumsum([0] + counts[:-1])
        have = [int(off[f:f + c].sum()) for f, c in zip(first, counts)]
        for src, walker, dst, n in plan:
            assert n > 0 and walker < counts[src] and have[src] > counts[src] and have[dst] < counts[dst]
        out = list(have)
        for src, walker, dst, n in plan:
            out[src] -= n
            out[dst] += n
        assert out == counts                      # every rank ends with its own count
        assert plan == P.plan_walker_exchange(off, counts)  # deterministic: every rank plans the same


def test_one_rank_is_the_single_rank_comb():
    SM, props = _table(23, 3)
    r = 0.4137
    SM1, pr1 = P.population_control(None, SM, props, r)
    wo = O.Walkers(SM)
    wo.weight = props[P.WEIGHT].copy()
    wo.phase = props[1].copy()
    O.population_control(wo, r)
    assert np.array_equal(SM1, wo.SM) and np.array_equal(pr1[P.WEIGHT], wo.weight)
    assert np.array_equal(pr1[1], wo.phase)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, counts, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    SM, props = _table(sum(counts), 7)
    first = sum(counts[:rank])
    mine = slice(first, first + counts[rank])
    SMr, prr = P.population_control(dist, SM[mine], props[:, mine], 0.27)
    q.put((rank, SMr, prr))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("counts", [[9, 9], [6, 11], [0, 12], [3, 10, 5], [7, 0, 9]])
def test_ranks_equal_one_rank_holding_everything(counts):
    """The walkers two or three gloo ranks end with are, together, the population one rank ends with,
    and each rank keeps its own count; the weights become unit-modulus."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = len(counts)
    procs = [ctx.Process(target=_rank, args=(r, world, port, counts, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    SM, props = _table(sum(counts), 7)
    SM1, pr1 = P.population_control(None, SM, props, 0.27)
    for rank, SMr, prr in out:
        assert SMr.shape[0] == counts[rank]
        assert np.allclose(np.abs(prr[P.WEIGHT]), 1.0)
    key = lambda S, pr: sorted(tuple(np.round(np.concatenate([S[i].ravel(), pr[:, i]]), 12)) for i in range(S.shape[0]))
    both = key(np.concatenate([o[1] for o in out]), np.concatenate([o[2] for o in out], axis=1))
    assert both == key(SM1, pr1)


def test_engine_with_back_propagation_is_refused():
    """Sharded population control moves only the Slater matrices and properties: an engine that keeps
    back-propagation history (fields, weight factors, anchors per walker) is refused before any
    walker is read or any message is sent."""
    class FakeEngine:
        nbp = 4

        def walkers(self):
            raise AssertionError("the walkers must not be read")

        properties = walkers

    with pytest.raises(capi.SafireError) as ei:
        P.engine_population_control(None, FakeEngine(), 0.5)
    assert ei.value.code == 3
