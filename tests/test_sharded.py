"""run_afqmc over walkers sharded across ranks (safire_b200.sharded) on two gloo ranks, each stepping
its share of BH's walkers with an oracle-backed stand-in for the engine (the host logic under test is
the cross-rank part: the global Eshift relaxation, the global measurement and the global comb).

Without population control inside the run, two ranks with the global field stream split between
them must reproduce one rank holding every walker; with it, every rank keeps its walker count and
all ranks agree on Eshift and the measurements."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import afqmc_oracle as O
from oracle.mt19937 import HostRandomGenerator, split_seed
from safire_b200 import capi
from safire_b200 import sharded as S
from tests.golden_io import bh_snapshot

NW = 24  # global walkers (divisible by 2 and 3 ranks)
FIELDS = dict(zip(capi.PROPS, ("weight", "phase", "pseudo_eloc", "e1", "exx", "ej", "ovlp", "theta")))


class OracleEngine:
    """The engine calls run_sharded makes, on the oracle's walkers and propagator (test stand-in)."""

    def __init__(self, ham, nwalk, dt, target):
        self.ham, self.W, self.Nc, self.dt = ham, nwalk, ham.Nc, dt
        psi = ham.trial_walker()
        self.w = O.Walkers(np.broadcast_to(psi, (nwalk,) + psi.shape))
        self.E_init = O.init_walkers(ham, self.w)
        self.prop = O.Propagator(ham, dt)
        self.target = target

    def walkers(self):
        return self.w.SM.copy(), {k: getattr(self.w, f).copy() for k, f in FIELDS.items()}

    def set_walkers(self, SM, props):
        self.w.SM = np.array(SM)
        for k, f in FIELDS.items():
            setattr(self.w, f, np.array(props[k]))

    def properties(self):
        return {k: getattr(self.w, f).copy() for k, f in FIELDS.items()}

    # the walker-exchange rows, on the host: Slater matrix then the 8 properties
    exchange_device = torch.device("cpu")

    def walker_row_elems(self):
        return self.w.SM[0].size + len(FIELDS)

    def pack_walkers(self, slots, rows):
        v = rows.numpy().view(np.complex128)
        for r, i in enumerate(slots):
            v[r] = np.concatenate([self.w.SM[i].ravel(), [getattr(self.w, f)[i] for f in FIELDS.values()]])

    def unpack_walkers(self, slots, rows):
        v = rows.numpy().view(np.complex128)
        n = self.w.SM[0].size
        for r, i in enumerate(slots):
            self.w.SM[i] = v[r, :n].reshape(self.w.SM.shape[1:])
            for j, f in enumerate(FIELDS.values()):
                getattr(self.w, f)[i] = v[r, n + j]

    def copy_walkers(self, pairs, normalize=True):
        if normalize:
            self.w.weight = self.w.weight / np.abs(self.w.weight)
        for src, dst in pairs:
            self.w.SM[dst] = self.w.SM[src]
            for f in FIELDS.values():
                getattr(self.w, f)[dst] = getattr(self.w, f)[src]

    def propagate_host(self, Eshift, step, uniforms_host):
        self.prop.propagate(self.w, Eshift, step, target_population=self.target, uniforms=uniforms_host)

    def orthogonalize(self):
        self.prop.orthogonalize(self.w)

    def measure(self):
        return O.measure_energy(self.ham, self.w)


def _run(rank, world, pop_interval):
    snap = bh_snapshot()
    ham = O.Hamiltonian(snap["hcore"], snap["Likn"], snap["PsiT"], snap["E0"])
    share = NW // world
    eng = OracleEngine(ham, share, 0.01, NW)
    field = HostRandomGenerator(split_seed(11, 0, 1))    # one global field stream, split by rank
    comb = HostRandomGenerator(split_seed(11, 0, 0))

    def uniforms(n):
        u = field.uniforms(NW * ham.Nc).reshape(NW, ham.Nc)
        return u[rank * share:(rank + 1) * share]

    dist = None
    if world > 1:
        import torch.distributed as dist
    Eshift, meas = S.run_sharded(dist, eng, 8, eng.E_init, lambda: comb.uniforms(1)[0], uniforms,
                                 ortho_interval=3, pop_interval=pop_interval, equilibration_steps=4,
                                 measure_interval=2, step0=1)
    return Eshift, meas, eng.W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, pop_interval, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    q.put((rank,) + _run(rank, world, pop_interval))
    dist.barrier()
    dist.destroy_process_group()


def _ranks(world, pop_interval):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, pop_interval, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_without_exchange_equal_one_rank(world):
    out = _ranks(world, pop_interval=1000)
    E1, m1, _ = _run(0, 1, 1000)
    for _, Eshift, meas, _ in out:
        assert abs(Eshift - E1) < 1e-10 * abs(E1)
        assert [s for s, _ in meas] == [s for s, _ in m1]
        for (_, a), (_, b) in zip(meas, m1):
            for k in ("Energy", "OnebodyEnergy", "ExchangeEnergy", "CoulombEnergy", "TotalWeight"):
                assert abs(a[k] - b[k]) < 1e-10 * max(1.0, abs(b[k])), k


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_with_exchange_agree_and_keep_their_counts(world):
    out = _ranks(world, pop_interval=2)
    (_, E_a, m_a, w_a) = out[0]
    for _, E_b, m_b, w_b in out:
        assert w_b == NW // world
        assert E_a == E_b and m_a == m_b               # every rank sees the global reductions
    assert all(np.isfinite(m["Energy"].real) for _, m in m_a)
    assert all(abs(m["TotalWeight"].real - NW) < 1e-9 for s, m in m_a if (s % 2) == 0)  # after a comb
