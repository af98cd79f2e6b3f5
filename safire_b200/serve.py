"""The serving loop (sfq_server_*): resident systems, requests that are propagation blocks,
continuous batching on the GPU; and its benchmark.

    python -m safire_b200.serve            # 40 systems, Poisson arrivals, p50/p99 block latency

The benchmark builds 40 synthetic systems (M uniform in [32, 400] on a multiple of 16, N = M/4,
Nchol = 6M, 128 walkers each, INT8X3 precision as the headline's), measures batch-mode capacity in a
steady state (many rounds of blocks of every system submitted at once and drained, so the tail of
the last blocks is a small part of the time), then drives Poisson arrivals at fractions of that
capacity, each request a block of 20 steps plus one local-energy measurement for a uniformly chosen
system, a fixed number of requests per rate (1000 by default, so that p99 is a percentile and not
the maximum), and prints one JSON line with p50/p99 block latency and walker-steps/s per rate.
"""
import argparse
import ctypes
import json
import time

import numpy as np

from . import capi, synthetic
from .capi import check, lib

# a block: 20 steps (orthogonalization every 5, population control every 20) and one measurement;
# Eshift is steered every step (the systems keep running block after block)
BLOCK = dict(ortho_interval=5, pop_interval=20, equilibration_steps=0, measure_interval=20, steer=True,
             relax=0.09516258196404048)  # 1 - exp(-10/100), run_afqmc's factor for 100 equilibration steps


class Server:
    def __init__(self, hbm_budget_gb=150.0, max_inflight=8, device=0):
        p = capi.ServerParams(int(hbm_budget_gb * 1e9), int(max_inflight), int(device))
        h = ctypes.c_void_p()
        check(lib().sfq_server_create(ctypes.byref(h), ctypes.byref(p)))
        self.h = h
        self.walkers = {}

    def close(self):
        if self.h:
            lib().sfq_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_system(self, system, nwalk, dt=0.005, seed=0, **params):
        ci = getattr(system, "ci", None)
        if ci is not None and np.size(ci) > 1:
            raise capi.SafireError(3, "the serving loop takes single-determinant systems; use AfqmcEngine "
                                      "(sfq_engine_create_nomsd) for a multi-determinant trial")
        p = capi.system_params(system, nwalk=nwalk, dt=dt, E0=float(system.E0), seed=seed)
        for k, v in params.items():
            setattr(p, k, v)
        h = np.ascontiguousarray(system.hcore, dtype=np.float64)
        L = np.ascontiguousarray(system.Likn, dtype=np.float64)
        P = np.ascontiguousarray(system.PsiT, dtype=np.complex128)
        sid = ctypes.c_int()
        check(lib().sfq_server_add_system(self.h, ctypes.byref(p), h.ctypes.data, L.ctypes.data, P.ctypes.data,
                                          ctypes.byref(sid)))
        self.walkers[sid.value] = nwalk
        return sid.value

    def warm(self, sid):
        check(lib().sfq_server_warm(self.h, int(sid)))

    def submit(self, sid, steps=20, ortho_interval=5, pop_interval=20, equilibration_steps=0, measure_interval=20,
               relax=0.0, steer=False):
        rp = capi.RunParams(steps, ortho_interval, pop_interval, equilibration_steps, measure_interval, relax, 0,
                            int(steer))
        rid = ctypes.c_longlong()
        check(lib().sfq_server_submit(self.h, int(sid), ctypes.byref(rp), ctypes.byref(rid)))
        return rid.value

    def progress(self):
        n = ctypes.c_int()
        check(lib().sfq_server_progress(self.h, ctypes.byref(n)))
        return n.value

    def request(self, rid):
        inf = capi.RequestInfo()
        meas = np.zeros((64, 10), np.float64)
        check(lib().sfq_server_request(self.h, int(rid), ctypes.byref(inf), meas.ctypes.data, 64))
        return {"status": inf.status, "system": inf.system, "t_submit": inf.t_submit, "t_start": inf.t_start,
                "t_finish": inf.t_finish, "Eshift": inf.Eshift, "step0": inf.step0, "meas": meas[:inf.nmeas].copy(),
                "message": inf.message.decode(errors="replace")}

    def stats(self):
        b, r, run, q = ctypes.c_size_t(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().sfq_server_stats(self.h, ctypes.byref(b), ctypes.byref(r), ctypes.byref(run), ctypes.byref(q)))
        return {"used_bytes": b.value, "resident": r.value, "running": run.value, "queued": q.value}

    def clock(self):
        return lib().sfq_server_clock(self.h)

    def drain(self, rids=None, timeout=600.0, poll=0.0001):
        """progress() until nothing is queued or running."""
        t0 = time.time()
        while True:
            self.progress()
            st = self.stats()
            if st["running"] == 0 and st["queued"] == 0:
                return
            if time.time() - t0 > timeout:
                raise TimeoutError(f"{st['running']} running, {st['queued']} queued")
            time.sleep(poll)


def _systems(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        M = int(rng.uniform(32, 400)) // 16 * 16
        M = max(M, 32)
        N = M // 4
        spec = synthetic.SystemSpec(M=M, N=N, Nc=6 * M, decay=float(M), seed=100 + i)
        out.append(synthetic.make_system(spec))
    return out


def system_dt(M):
    """Timestep of a serving system: these synthetic systems' force bias grows as the walkers move
    away from the (poor) trial, and the walkers of the larger ones die out after a few hundred steps
    at dt = 5e-4; with dt = 5e-5 * 256 / M every system (M = 48 .. 400, 128 walkers) survives 250
    blocks of 20 steps, the benchmark's length, while 1e-4 * 256 / M lost M = 320 and 400 after 60-70
    blocks.  The work per step does not depend on dt."""
    return float(min(max(5e-5 * 256.0 / M, 2.5e-5), 5e-4))


def _percentile(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=40)
    ap.add_argument("--walkers", type=int, default=128)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--inflight", type=int, default=8)
    ap.add_argument("--rates", default="0.1,0.3,0.5,0.7,0.9,1.0,1.2")
    ap.add_argument("--requests", type=int, default=1000, help="requests per rate")
    ap.add_argument("--batch-rounds", type=int, default=12)
    ap.add_argument("--precision", default="int8x3", choices=["int8x3", "mixed", "fp64"])
    a = ap.parse_args()
    prec = {"int8x3": capi.PRECISION_INT8X3, "mixed": capi.PRECISION_MIXED, "fp64": capi.PRECISION_FP64}[a.precision]
    systems = _systems(a.systems, 7)
    srv = Server(a.budget_gb, a.inflight)
    ids = [srv.add_system(s, a.walkers, dt=system_dt(s.M), seed=1000 + i, precision=prec)
           for i, s in enumerate(systems)]
    t0 = time.time()
    for sid in ids:
        srv.warm(sid)
    build_s = time.time() - t0
    blk = dict(BLOCK, steps=a.steps)
    # one warm block per system (graph capture), then batch mode: batch_rounds blocks of every system
    # submitted at once and drained (the server runs them max_inflight at a time)
    srv.drain([srv.submit(sid, **blk) for sid in ids])
    t0 = srv.clock()
    srv.drain([srv.submit(sid, **blk) for _ in range(a.batch_rounds) for sid in ids])
    batch_s = srv.clock() - t0
    nblocks = a.batch_rounds * len(ids)
    ws_block = a.walkers * a.steps
    batch_ws = nblocks * ws_block / batch_s
    cap_rps = nblocks / batch_s  # blocks per second at capacity
    rng = np.random.default_rng(11)
    rows = []
    for f in [float(x) for x in a.rates.split(",")]:
        lam = f * cap_rps
        arrivals = np.cumsum(rng.exponential(1.0 / lam, size=a.requests))
        # every system equally often, in random order: the same mix of block sizes as the batch run
        # (uniform random picks leave a few per cent of the work to chance at 1000 requests)
        picks = rng.permutation(np.resize(np.arange(len(ids)), len(arrivals)))
        rids = []
        base = srv.clock()
        k = 0
        while k < len(arrivals):
            now = srv.clock() - base
            while k < len(arrivals) and arrivals[k] <= now:
                rids.append(srv.submit(ids[picks[k]], **blk))
                k += 1
            srv.progress()
            time.sleep(0.0001)
        srv.drain()
        info = [srv.request(r) for r in rids]
        lat = [i["t_finish"] - i["t_submit"] for i in info if i["status"] == 0]
        span = max(i["t_finish"] for i in info) - base if info else 1.0
        rows.append({"load": f, "requests": len(info), "p50_ms": 1e3 * _percentile(lat, 50),
                     "p99_ms": 1e3 * _percentile(lat, 99), "walker_steps_per_s": len(lat) * ws_block / span,
                     "fraction_of_batch": len(lat) * ws_block / span / batch_ws,
                     "failed": sum(1 for i in info if i["status"] != 0),
                     "errors": sorted({i["message"][:100] for i in info if i["status"] != 0})[:3]})
    st = srv.stats()
    srv.close()
    print(json.dumps({
        "metric": "serving block latency", "unit": "ms", "systems": len(ids), "walkers_per_system": a.walkers,
        "block": f"{a.steps} steps + 1 local-energy measurement", "precision": a.precision,
        "requests_per_rate": a.requests, "batch_blocks": nblocks,
        "dt": "5e-5 * 256 / M, clipped to [2.5e-5, 5e-4]", "max_inflight": a.inflight, "hbm_budget_gb": a.budget_gb, "resident_bytes": st["used_bytes"],
        "build_seconds": build_s, "batch_walker_steps_per_s": batch_ws, "batch_blocks_per_s": cap_rps,
        "rates": rows, "data": "synthetic (M uniform in [32, 400] on multiples of 16, N = M/4, Nchol = 6M)"}))


if __name__ == "__main__":
    main()
