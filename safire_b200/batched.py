"""Several uneven systems advanced together, against the same systems one at a time in FP64.

    python -m safire_b200.batched        # 24 systems, M = 48, 64, ..., 320 (cycled), N = M/4,
                                         # Nchol = 5M, walkers log-uniform in [64, 512]

Every system gets a resident engine of the chosen precision (default INT8X3: int8-slice products
with exact integer accumulation; `--precision mixed-fp32`: 3 BF16 planes, its tile widths chosen
by the autotuner, sfq_engine_autotune), the LU / log det / QR / weights in FP64.  The engines form
one group (sfq_group_*): one block of every system is one CUDA graph launch, scheduled either fused
(INT8X3: the systems' steps stage by stage, each stage's tensor-core products of all systems as ONE
grouped launch) or in lanes that run side by side (members of a lane in turn), the schedule picked
by timing real blocks (EngineGroup.tune_lanes).  The block is 20
steps (orthogonalization every 5, population control and one local-energy measurement at the end,
Eshift steered every step).  Three timings of the same blocks:

  group          all systems per graph launch (host clock around K blocks, each ending with its
                 results on the host)
  mixed_serial   the same engines one at a time (sfq_engine_block), summed
  fp64_serial    FP64 engines one at a time, summed: the systems run one at a time with the FP64
                 drop-in

Accuracy per system, from identical walkers and seeded fields: one step of the mixed and the FP64
engine (relative error of fields, walkers, log overlaps, weights, local energies) and the weighted
local energy of the same walkers.  One JSON line.
"""
import argparse
import json
import math
import time

import numpy as np

from . import capi, synthetic
from .afqmc import AfqmcEngine, EngineGroup
from .serve import BLOCK, system_dt


def uneven_specs(count=24, seed=5):
    """M = 48, 64, ..., 320 cycled, N = M/4, Nchol = 5M; walkers log-uniform in [64, 512]."""
    rng = np.random.default_rng(seed)
    specs, walkers = [], []
    for i in range(count):
        M = 48 + 16 * (i % 18)
        specs.append(synthetic.SystemSpec(M=M, N=M // 4, Nc=5 * M, decay=float(M), seed=300 + i))
        walkers.append(int(round(math.exp(rng.uniform(math.log(64), math.log(512))))))
    return specs, walkers


def _make_engine(spec, W, seed, precision):
    return AfqmcEngine(synthetic.make_system(spec), W, dt=system_dt(spec.M), seed=seed, precision=precision)


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _accuracy(eng, eng64, W, spec, Eshift, step):
    """Identical walkers in both engines: the weighted local energy, then one step of both."""
    SM, pr = eng64.walkers()
    eng.set_walkers(SM, pr)
    dE = eng.measure()["Energy"].real - eng64.measure()["Energy"].real
    eng.propagate(Eshift, step)
    eng64.propagate(Eshift, step)
    X = eng.fetch("X", (W, spec.Nc), np.complex128)
    X64 = eng64.fetch("X", (W, spec.Nc), np.complex128)
    S, p = eng.walkers()
    S64, p64 = eng64.walkers()
    E, E64 = eng.energy(), eng64.energy()
    return {"energy_same_walkers_mHa": 1e3 * dE, "fields": _rel(X.imag, X64.imag), "walkers": _rel(S, S64),
            "log_overlap": _rel(p["OVLP"], p64["OVLP"]), "weights": _rel(p["WEIGHT"], p64["WEIGHT"]),
            "local_energy": _rel(E.sum(1), E64.sum(1))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=24)
    ap.add_argument("--steps", type=int, default=20, help="steps per block")
    ap.add_argument("--blocks", type=int, default=3, help="timed blocks")
    ap.add_argument("--warmup", type=int, default=2, help="untimed blocks per timing (the first captures graphs)")
    ap.add_argument("--lanes", default="fused,1,2,3,4,6,8,0",
                    help="schedules the tuner tries: 'fused' (int8-slice precisions: each stage's products of all "
                         "systems as one grouped launch) and lane counts (0: one lane per system)")
    ap.add_argument("--no-tune", action="store_true", help="keep the built-in tiles")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--precision", default="int8x3", choices=["int8x3", "mixed-fp32", "mixed"])
    a = ap.parse_args()
    specs, walkers = uneven_specs(a.systems)
    blk = dict(ortho_interval=BLOCK["ortho_interval"], pop_interval=a.steps, equilibration_steps=0,
               measure_interval=a.steps, relax=BLOCK["relax"], steer=True)
    prec = {"int8x3": capi.PRECISION_INT8X3, "mixed-fp32": capi.PRECISION_MIXED_FP32,
            "mixed": capi.PRECISION_MIXED}[a.precision]
    tunable = True  # split-BF16: every product's width; int8 slices: the Taylor term's orbitals per tile

    # resident mixed engines, autotuned
    t0 = time.time()
    engines, Esh, tiles, tune = [], [], [], {"us_builtin": 0.0, "us_tuned": 0.0}
    for i, (spec, W) in enumerate(zip(specs, walkers)):
        e = _make_engine(spec, W, 1000 + i, prec)
        Esh.append(e.init())
        if tunable and not a.no_tune:
            t = e.autotune()
            tiles.append(t.choice())
            w = (1, 1, 1, 6, 1)  # per step: G, vbias, vHS, six Taylor terms, the P1 pair
            tune["us_builtin"] += sum(w[k] * t.us_builtin[k] for k in range(5))
            tune["us_tuned"] += sum(w[k] * t.us_tuned[k] for k in range(5))
        else:
            tiles.append(e.tiles())
        engines.append(e)
    build_s = time.time() - t0
    foot = sum(e.footprint() for e in engines)
    init_state = [e.walkers() for e in engines]
    Esh0 = list(Esh)
    ws_block = sum(walkers) * a.steps

    # the same engines one at a time, from their initial walkers
    serial_s = 0.0
    for i, e in enumerate(engines):
        E = Esh0[i]
        s0 = 0
        for _ in range(a.warmup):
            E, _m = e.run_block(a.steps, E, step0=s0, **blk)
            s0 += a.steps
        e.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.blocks):
            E, _m = e.run_block(a.steps, E, step0=s0, **blk)
            s0 += a.steps
        serial_s += time.perf_counter() - t0
        e.set_walkers(*init_state[i])

    # group: all systems per graph launch; the lane count from timed real blocks
    grp = EngineGroup(engines)
    es = np.asarray(Esh0, np.float64)
    step0 = 0
    lane_times = {}
    cands = [x if x == "fused" else int(x) for x in a.lanes.split(",")]
    if a.precision != "int8x3":
        cands = [c for c in cands if c != "fused"]
    if len(cands) > 1:
        es, step0, lane_times = grp.tune_lanes(a.steps, es, step0=step0, candidates=cands, **blk)
    else:
        grp._schedule(cands[0])
    for _ in range(a.warmup):
        es, st, _m = grp.run_block(a.steps, es, step0=step0, **blk)
        step0 += a.steps
    t0 = time.perf_counter()
    for _ in range(a.blocks):
        es, st, _m = grp.run_block(a.steps, es, step0=step0, **blk)
        step0 += a.steps
    group_s = time.perf_counter() - t0
    lanes = "fused" if grp.fused else grp.lanes
    grp.close()

    # FP64 engines one at a time: timing, then accuracy against the mixed engine
    fp64_s, acc = 0.0, []
    if not a.no_fp64:
        for i, (spec, W) in enumerate(zip(specs, walkers)):
            e64 = _make_engine(spec, W, 1000 + i, capi.PRECISION_FP64)
            E = e64.init()
            s0 = 0
            for _ in range(max(1, a.warmup - 1)):
                E, _m = e64.run_block(a.steps, E, step0=s0, **blk)
                s0 += a.steps
            e64.synchronize()
            t0 = time.perf_counter()
            for _ in range(a.blocks):
                E, _m = e64.run_block(a.steps, E, step0=s0, **blk)
                s0 += a.steps
            fp64_s += time.perf_counter() - t0
            acc.append(dict(M=spec.M, W=W, **_accuracy(engines[i], e64, W, spec, E, s0)))
            e64.close()
    for e in engines:
        e.close()

    def rate(sec):
        return a.blocks * ws_block / sec if sec > 0 else None

    out = {
        "metric": "walker-steps/s", "unit": "walker-steps/s",
        "workload": f"{len(specs)} systems, M = 48..320 step 16 cycled, N = M/4, Nchol = 5M, walkers log-uniform "
                    f"[64, 512] (total {sum(walkers)}); blocks of {a.steps} steps (ortho every "
                    f"{blk['ortho_interval']}, population control + 1 measurement per block, steered Eshift)",
        "systems": [{"M": s.M, "N": s.N, "Nc": s.Nc, "W": w} for s, w in zip(specs, walkers)],
        "precision": {"int8x3": "int8 slices x3 (exact int32 accumulation)", "mixed-fp32": "3 BF16 planes",
                      "mixed": "2 BF16 planes"}[a.precision] + "; LU/log det/QR/weights FP64",
        "group": {"value": rate(group_s), "ms_per_block": 1e3 * group_s / a.blocks, "lanes": lanes,
                  "lane_seconds_per_block": {str(k): v for k, v in lane_times.items()},
                  "how": "one CUDA graph per block; 'fused': the members' steps stage by stage, each stage's "
                         "int8-slice products of all members as one grouped launch; else members in `lanes` "
                         "chains side by side (0: one per member)"},
        "mixed_serial": {"value": rate(serial_s), "ms_per_block": 1e3 * serial_s / a.blocks},
        "fp64_serial": {"value": rate(fp64_s), "ms_per_block": 1e3 * fp64_s / a.blocks} if fp64_s else None,
        "speedup_group_vs_fp64_serial": fp64_s / group_s if fp64_s else None,
        "speedup_group_vs_mixed_serial": serial_s / group_s,
        "autotune": {"tiles": tiles, "step_products_us_builtin": tune["us_builtin"],
                     "step_products_us_tuned": tune["us_tuned"]} if not a.no_tune else None,
        "accuracy": acc, "max_abs_energy_same_walkers_mHa": max((abs(r["energy_same_walkers_mHa"]) for r in acc),
                                                                default=None),
        "resident_bytes": foot, "build_seconds": build_s, "dt": "5e-5 * 256 / M, clipped to [2.5e-5, 5e-4]",
        "data": "synthetic (seeded random Cholesky tensors and trial)",
        "timing": "host clock around the timed blocks, each ending with its results on the host",
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
