"""Several GPUs of one node run independent replicas (no collective on the data path): the job's
time is the maximum over ranks and its throughput every rank's walker-steps over that time.  Two
gloo ranks on the CPU exercise the same host logic bench.py runs under torchrun."""
import os
import socket

import torch.multiprocessing as mp

from safire_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist = replicas.init(world, backend="gloo", timeout_s=60)
    ms = replicas.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")  # the slower rank's time wins
    q.put((rank, ms, replicas.job_rate(256 * 20, world, ms), replicas.seed_for(rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]                   # max over ranks on every rank
    assert out[0][2] == out[1][2] == 256 * 20 * 2 / 15e-3       # whole-job walker-steps/s
    assert out[0][3] != out[1][3]                                # independent walker populations


def test_one_rank_needs_no_group():
    assert replicas.init(1) is None
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_rate(100, 1, 10.0) == 1e4
