#!/usr/bin/env python
"""Walker-steps/s of the AFQMC propagation path on B200 (one JSON line on rank 0).

A "step" is one iteration of run_afqmc's loop in its equilibration phase: Propagate of every
walker (force bias, fields, vHS, P1 + order-6 Taylor exp, overlap, walker update, weight bound),
orthogonalization every 5 steps and comb population control every 20 steps amortised into the
steps they fall on, and the Eshift relaxation from the growth estimator.  Workload (default): synthetic dense-Cholesky
system M=400, N=100+100 (closed shell), Nchol=2400, 256 walkers, dt=0.0005, Philox fields, the
products from int8 slices with exact accumulation (INT8X3), against the FP64 drop-in in the same run.

  value       device time (CUDA events on the engine stream), inputs resident in HBM
  e2e         the same steps through sfq_engine_propagate_host: the step's field uniforms are
              copied from pinned host memory and the walker properties read back every step
  roofline    the dominant kernel (one Taylor-term product) timed with CUDA events inside this run
  cpu_baseline the FP64 oracle (numpy + LAPACK/BLAS) on a bounded walker sample, on host cores

--impl reference times the CPU restatement of the reference's path (the oracle) on the same
configuration, walkers split over all host threads with one BLAS thread each.  Under torchrun every rank runs an independent walker
population of the same system (replicas; weak scaling); timings are max over ranks.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# dt: the small system uses the configured 0.005.  With the same tensor distributions, M=128 and
# M=400 give |vHS| ~ 1.1 and ~ 2 per step at dt = 0.005 and the phaseless constraint zeroes every
# walker within a few steps (the oracle shows it; the reference's comb then aborts), so those
# systems run at the dt where |vHS| ~ 0.5-0.7 per step.  The work per step does not depend on dt.
CONFIGS = {
    "large": dict(spec="CFG_LARGE", nwalk=256, cpu_walkers=64, dt=0.0005),
    "medium": dict(spec="CFG_MEDIUM", nwalk=1024, cpu_walkers=64, dt=0.002),
    "small": dict(spec="CFG_SMALL", nwalk=32, cpu_walkers=32, dt=0.005),
}
ORTHO_EVERY = 5
POP_EVERY = 20
# DRAM bytes (read + write) of one Taylor-term int8 product at 256 walkers, M = 400, N = 100, from an
# ncu capture of the same kernel and tile (profiles/islice_taylor_M400_N100_W256_full.md)
TAYLOR_DRAM_BYTES_256 = 485.248512e6 + 68.982528e6
EQUIL_STEPS = 100  # run_afqmc relaxes Eshift every step for the first equilibration_steps
RELAX = 1.0 - math.exp(-10.0 / EQUIL_STEPS)


def step_flops(M, N, Nc):
    """Algorithmic flops per walker-step (complex multiply-add = 8 real flops)."""
    return 8 * N * M * Nc + 4 * M * M * Nc + 64 * M * M * N + 24 * N * N * M + (32 / 3) * N ** 3


def taylor_flops(M, N, W):
    """Algorithmic flops of one Taylor-term launch: every walker's complex (M x M) vHS times its
    complex (M x N) term, 8 real flops per complex multiply-add."""
    return 8.0 * M * M * N * W


def vhs_flops(M, Nc, W, packed):
    """Algorithmic flops of one vHS launch: real L (M^2 x Nc, or its M(M+1)/2 packed upper-triangle
    rows when the Cholesky vectors are symmetric) times complex X (Nc x W)."""
    rows = M * (M + 1) // 2 if packed else M * M
    return 4.0 * rows * Nc * W


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.lines = []
        self.dev = device_index

    def start(self):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            sel = ["-i", uuid if uuid.startswith("GPU-") else "GPU-" + uuid]
        except Exception:
            sel = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200"] + sel, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def fp64_gemm_peak_tflops(dev):
    """cuBLAS DGEMM throughput on this GPU (FP64 has no driver-measured peak)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e30
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


L2_BYTES = 126e6  # B200 L2


def l2_note(spec, nwalk):
    """Whether a step's inputs (the Cholesky tensor and the walkers' Slater matrices) outgrow L2, so
    that no flush is needed between timed steps, or fit in it."""
    likn = spec.M ** 2 * spec.Nc * 8
    walkers = nwalk * spec.M * spec.N * 16
    if likn + walkers > L2_BYTES:
        return "inputs larger than L2 (Likn %.2f GB + walkers %.2f GB)" % (likn / 1e9, walkers / 1e9)
    return "inputs fit in L2 (Likn %.4f GB + walkers %.4f GB), not flushed between steps" % (
        likn / 1e9, walkers / 1e9)


def workload_config(cfg, spec, precision, world):
    """The workload both arms report (the same dict, so their lines describe the same config)."""
    return {"workload": f"AFQMC propagation {spec.name}: dense real Cholesky, closed shell, "
                        f"{cfg['nwalk']} walkers per GPU",
            "M": spec.M, "N": spec.N, "Nchol": spec.Nc, "walkers_per_gpu": cfg["nwalk"], "dt": cfg["dt"],
            "precision": precision, "eshift": "relaxed every step (equilibration phase of run_afqmc)",
            "taylor_order": 6, "ortho_every": ORTHO_EVERY, "popcontrol_every": POP_EVERY,
            "l2": l2_note(spec, cfg["nwalk"]),
            "parallelism": f"replicas x{world}"}


def cpu_port_rate(cfg, steps=5, warm=2, walkers=None, with_popcontrol=False):
    """The FP64 oracle (numpy/LAPACK restatement of the reference path) on a bounded walker sample of
    the same system, as the reference runs on CPUs: walkers split over one worker per host core
    (execute.cpp:140, one thread per rank), each worker's BLAS on one thread
    (threading.cpp:27-36).  2 warm-up steps, then `steps` timed steps (orthogonalization every 5,
    Eshift relaxed; with with_popcontrol, the comb at the GPU arm's interval, each worker's shard
    combed on its own)."""
    import concurrent.futures as cf
    from threadpoolctl import threadpool_limits
    from oracle import afqmc_oracle as O
    from oracle import philox
    from safire_b200 import synthetic
    spec = getattr(synthetic, cfg["spec"])
    s = synthetic.make_system(spec)
    Ws = walkers or cfg["cpu_walkers"]
    cores = os.cpu_count() or 1
    nthr = max(1, min(cores, Ws))
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    dt = cfg["dt"]
    shards = [Ws // nthr + (1 if r < Ws % nthr else 0) for r in range(nthr)]
    props = [O.Propagator(ham, dt, seed=r) for r in range(nthr)]
    wsets = [O.Walkers(s.initial_walkers(n)) for n in shards]
    Esh = [O.init_walkers(ham, w) for w in wsets]

    def shard_step(r, st):
        props[r].propagate(wsets[r], Esh[r], st)
        if st % ORTHO_EVERY == 0:
            props[r].orthogonalize(wsets[r])
        Esh[r] += RELAX * (O.average_pseudo_energy(wsets[r], dt) - Esh[r])

    with threadpool_limits(limits=1), cf.ThreadPoolExecutor(max_workers=nthr) as ex:
        def step(st):
            list(ex.map(lambda r: shard_step(r, st), range(nthr)))
            if with_popcontrol and st % POP_EVERY == 0:
                for r in range(nthr):
                    O.population_control(wsets[r], philox.comb_uniform(r, st))

        for st in range(warm):
            step(st)
        t0 = time.perf_counter()
        for st in range(warm, warm + steps):
            step(st)
        t = time.perf_counter() - t0
    return dict(value=Ws * steps / t, unit="walker-steps/s", cores=nthr, kind="port",
                sample=f"{Ws} walkers of {spec.name} split over {nthr} host threads (BLAS 1 thread each), "
                       f"{steps} timed steps after {warm} warm-up; FP64 numpy/LAPACK restatement of the "
                       "reference path", seconds=t)


def run_reference(args, cfg):
    """--impl reference: the reference's path on the host cores (the oracle port, since the reference
    itself cannot be built here), on the same workload; each step a bounded walker sample."""
    from safire_b200 import synthetic
    spec = getattr(synthetic, cfg["spec"])
    r = cpu_port_rate(cfg, steps=args.steps, warm=args.warmup, with_popcontrol=True)
    value, unit = r["value"], r["unit"]
    line = {"impl": "reference", "metric": "walker-steps/s", "value": value, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(cfg, spec, args.precision, args.gpus),
            "cpu_baseline": {"value": value, "unit": unit, "cores": r["cores"], "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def step_errors(eng, eng64, W, spec, Eshift, step):
    """One step of both engines from the FP64 engine's walkers with the same seeded fields: the
    relative error (max |mixed - fp64| / max |fp64|) of each quantity of the step."""
    import numpy as np

    def rel(a, b):
        a, b = np.asarray(a), np.asarray(b)
        return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))

    SM, pr = eng64.walkers()
    eng.set_walkers(SM, pr)
    eng.propagate(Eshift, step)
    eng64.propagate(Eshift, step)
    X = eng.fetch("X", (W, spec.Nc), np.complex128)
    X64 = eng64.fetch("X", (W, spec.Nc), np.complex128)
    S, p = eng.walkers()
    S64, p64 = eng64.walkers()
    E, E64 = eng.energy(), eng64.energy()
    return {"fields_from_vbias": rel(X.imag, X64.imag), "propagated_walkers": rel(S, S64),
            "log_overlap": rel(p["OVLP"], p64["OVLP"]), "weights": rel(p["WEIGHT"], p64["WEIGHT"]),
            "local_energy_E1": rel(E[:, 0], E64[:, 0]), "local_energy_EXX": rel(E[:, 1], E64[:, 1]),
            "local_energy_EJ": rel(E[:, 2], E64[:, 2]), "local_energy": rel(E.sum(1), E64.sum(1)),
            "how": "one step of both engines from identical walkers and seeded fields; max |mixed - fp64| / max |fp64|"}


def seeded_block_delta(s, W, DT, prec, seed, steps):
    """Block energy difference (mHa) of `prec` against the FP64 drop-in after `steps` steps of the
    benchmark's schedule from the same seed (untimed)."""
    from safire_b200 import afqmc, capi
    E = {}
    for p in (capi.PRECISION_FP64, prec):
        eng = afqmc.AfqmcEngine(s, W, dt=DT, seed=seed, device=0, precision=p)
        Esh = eng.init()
        for st in range(steps):
            eng.propagate(Esh, st)
            if st % ORTHO_EVERY == 0:
                eng.orthogonalize()
            if st % POP_EVERY == 0:
                eng.population_control(st)
            Esh += RELAX * (eng.averages()[0] - Esh)
        E[p] = eng.measure()["Energy"].real
        eng.close()
    return 1e3 * (E[prec] - E[capi.PRECISION_FP64])


def run_engine(args, cfg, spec, s, W, DT, prec, rank, local, profile_pass=True, e2e=True):
    """Warm up, time args.steps steps on the device, optionally a profile pass and the e2e pass.

    Returns (engine, dict of measurements); the engine is left open for the caller.
    """
    import torch
    from safire_b200 import afqmc, capi
    L = capi.lib()
    from safire_b200 import replicas
    eng = afqmc.AfqmcEngine(s, W, dt=DT, seed=replicas.seed_for(rank), device=local, precision=prec)
    state = {"Esh": eng.init()}
    ext = torch.cuda.ExternalStream(eng.stream)
    out = {}
    if prec != capi.PRECISION_FP64 and not getattr(args, "no_autotune", False):
        out["tiles"] = eng.autotune().choice()  # tile widths from timing the products on this engine

    def step(st, host=False, ubuf=None, pbuf=None):
        """One run_afqmc iteration in the equilibration phase (run_afqmc.cpp:69-93)."""
        if host:
            eng.propagate_host(state["Esh"], st, ubuf, pbuf)
        else:
            eng.propagate(state["Esh"], st)
        if st % ORTHO_EVERY == 0:
            eng.orthogonalize()
        if st % POP_EVERY == 0:
            eng.population_control(st)
        pe = eng.averages()[0]
        state["Esh"] += RELAX * (pe - state["Esh"])

    for st in range(args.warmup):
        step(st)
    eng.synchronize()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    n0 = L.sfq_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for st in range(args.warmup, args.warmup + args.steps):
        step(st)
    e1.record(ext)
    e1.synchronize()
    out["launches"] = int(L.sfq_launch_count() - n0)
    out["clocks"] = clk.stop()
    out["ms"] = e0.elapsed_time(e1)
    # energy at the end of the timed block (EnergyEstimator::measure), outside the timed region
    meas = eng.measure()
    out["energy"] = meas["Energy"].real
    s1 = args.warmup + args.steps
    if profile_pass:
        eng.profile(True)
        for st in range(s1, s1 + args.steps):
            step(st)
        out["phases"] = eng.phase_times()
        eng.profile(False)
        s1 += args.steps
    if e2e:
        ubytes = W * spec.Nc * 8
        pbytes = 8 * W * 16
        ubuf = torch.empty((args.steps, W, spec.Nc), dtype=torch.float64).pin_memory()
        pbuf = torch.empty((args.steps, 8, W), dtype=torch.complex128).pin_memory()
        tmp = torch.empty((W, spec.Nc), dtype=torch.float64, device="cuda")
        for i in range(args.steps):
            capi.check(L.sfq_field_uniforms(tmp.data_ptr(), replicas.seed_for(rank), s1 + i, W, spec.Nc, None))
            ubuf[i].copy_(tmp.cpu())
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        tw = time.perf_counter()
        f0.record(ext)
        for i in range(args.steps):
            step(s1 + i, host=True, ubuf=ubuf[i], pbuf=pbuf[i])
        f1.record(ext)
        f1.synchronize()
        wall = time.perf_counter() - tw
        out["e2e_ms"] = max(f0.elapsed_time(f1), wall * 1e3)
        out["e2e_bytes"] = (ubytes, pbytes)
    out["vhs_packed"] = bool(eng.info().vhs_packed)
    return eng, out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="large", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="int8x3", choices=["fp64", "int8x3", "int8x2", "mixed", "mixed-fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 drop-in comparison run")
    ap.add_argument("--no-autotune", action="store_true", help="keep the built-in tile widths")
    ap.add_argument("--compare-seeds", type=int, default=5,
                    help="further seeds for the block-energy comparison against FP64 (untimed)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    cfg = CONFIGS[args.config]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, cfg)
        return

    import torch
    from safire_b200 import capi, replicas, synthetic

    torch.cuda.set_device(local)
    dist = replicas.init(world, "nccl", timeout_s=300)

    spec = getattr(synthetic, cfg["spec"])
    W = cfg["nwalk"]
    DT = cfg["dt"]
    s = synthetic.make_system(spec)
    prec = {"fp64": capi.PRECISION_FP64, "mixed": capi.PRECISION_MIXED, "mixed-fp32": capi.PRECISION_MIXED_FP32,
            "int8x3": capi.PRECISION_INT8X3, "int8x2": capi.PRECISION_INT8X2}[args.precision]
    if dist:
        dist.barrier()
    eng, m = run_engine(args, cfg, spec, s, W, DT, prec, rank, local, e2e=not args.no_e2e)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, device="cuda")

    ms = max_over_ranks(m["ms"])
    value = replicas.job_rate(W * args.steps, world, ms)
    e2e = None
    if "e2e_ms" in m:
        ems = max_over_ranks(m["e2e_ms"])
        e2e = {"value": replicas.job_rate(W * args.steps, world, ems), "unit": "walker-steps/s",
               "h2d_bytes_per_step": m["e2e_bytes"][0], "d2h_bytes_per_step": m["e2e_bytes"][1],
               "path": "sfq_engine_propagate_host (pinned host uniforms in, walker properties out)"}

    # the FP64 drop-in on the same system, seeds and schedule: speed ratio and block-energy difference
    compare = None
    if prec != capi.PRECISION_FP64 and not args.no_compare:
        eng64, m64 = run_engine(args, cfg, spec, s, W, DT, capi.PRECISION_FP64, rank, local, profile_pass=False,
                                e2e=False)
        errors = step_errors(eng, eng64, W, spec, m64["energy"], args.warmup + args.steps + 1000)
        eng64.close()
        del eng64
        ms64 = max_over_ranks(m64["ms"])
        v64 = replicas.job_rate(W * args.steps, world, ms64)
        compare = {"fp64_value": v64, "fp64_ms_per_step": ms64 / args.steps, "speedup_vs_fp64": value / v64,
                   "block_energy_mixed": m["energy"], "block_energy_fp64": m64["energy"],
                   "block_energy_delta_mHa": 1e3 * (m["energy"] - m64["energy"]),
                   "block_energy_delta_rel": (m["energy"] - m64["energy"]) / abs(m64["energy"]),
                   "block": f"energy measured after the {args.warmup}+{args.steps} steps of each timed run",
                   "step_errors": errors}
        if args.compare_seeds > 0 and rank == 0:
            # the same comparison from further seeds (untimed): the fixed-point slices' noise moves
            # one seeded block either way; a bias would show in the mean
            ds = [compare["block_energy_delta_mHa"]]
            for sd in range(1, args.compare_seeds + 1):
                ds.append(seeded_block_delta(s, W, DT, prec, sd, args.warmup + args.steps))
            d = np.array(ds)
            compare["seeds"] = {"seeds": [replicas.seed_for(rank)] + list(range(1, args.compare_seeds + 1)),
                                "block_energy_delta_mHa": [float(x) for x in d],
                                "mean_mHa": float(d.mean()),
                                "sem_mHa": float(d.std(ddof=1) / math.sqrt(len(d))),
                                "max_abs_mHa": float(np.max(np.abs(d)))}
    eng.close()
    del eng

    # ---- roofline of the dominant kernel: the Taylor-term product --------------------------
    ph = m["phases"]
    peaks = measured_peaks()
    t_ms, t_n = ph["taylor_gemm"]
    launch_ms = t_ms / max(t_n, 1)
    alg = taylor_flops(spec.M, spec.N, W)
    achieved = alg / (launch_ms * 1e-3) / 1e12
    v_ms, v_n = ph["vHS_gemm"]
    v_launch = v_ms / max(v_n, 1)
    v_alg = vhs_flops(spec.M, spec.Nc, W, m["vhs_packed"])
    if prec == capi.PRECISION_FP64:
        peak = fp64_gemm_peak_tflops(local)
        roofline = {"bound": "tensor", "kernel": "gemm_f64_kernel (Taylor term: complex vHS x complex walkers, DMMA)",
                    "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (no FP64 entry in the peaks file)"}
    else:
        peak = peaks.get("bf16_tflops_sustained") or 1400.0
        src = ("MEASURED_PEAKS.json bf16_tflops_sustained, of measured (kernel timed inside a long step)"
               if peaks.get("bf16_tflops_sustained") else "fallback 1.4 PFLOP/s sustained")
        if prec in (capi.PRECISION_INT8X3, capi.PRECISION_INT8X2):
            ns = 3 if prec == capi.PRECISION_INT8X3 else 2
            npairs = 6 if ns == 3 else 3
            # the complex product runs as [re|im] += A_re [Vr;Vi]^T, re += (-A_im) Vi^T, im += A_im Vr^T:
            # 2 real products' worth of work per complex one, times the slice pairs, on rows padded
            # to 128 and orbitals to the tile
            rows = 128 * ((spec.N + 127) // 128)
            kpad = 32 * ((spec.M + 31) // 32)
            executed = 2.0 * 2 * rows * (2 * spec.M) * kpad * W * npairs
            roofline = {"bound": "tensor",
                        "kernel": f"islice_gemm_kernel (Taylor term: int8 slices x{ns}, tcgen05 kind::i8, exact "
                                  f"int32 accumulation, {npairs} int8 products per real product)",
                        "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                        "executed_int8_tops": executed / (launch_ms * 1e-3) / 1e12,
                        "executed_frac_of_int8": executed / (launch_ms * 1e-3) / 1e12 / (2 * peak),
                        "int8_peak_note": "int8 tensor rate taken as twice the measured bf16 rate (B200's ratio)",
                        "peak_source": src}
        else:
            nprod = 3 if prec == capi.PRECISION_MIXED else 6
            roofline = {"bound": "tensor",
                        "kernel": f"umma_gemm_kernel (Taylor term: split-BF16 tcgen05, {nprod} tensor-core products "
                                  "per real product)",
                        "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                        "executed_tflops": achieved * nprod * 2, "peak_source": src}
    traffic = None
    if prec == capi.PRECISION_INT8X3 and spec.M == 400 and spec.N == 100:
        # dram__bytes_read.sum + dram__bytes_write.sum of the Taylor product in one ncu capture of
        # sfq_gemm_int8_cplx_b at 256 walkers, M = 400, N = 100 (the same kernel and tile), scaled
        # to this launch's walkers: every byte moved is per walker
        traffic = TAYLOR_DRAM_BYTES_256 * W / 256.0
        roofline.update({"traffic_unit": "bytes per launch",
                         "traffic_source": "ncu capture of the same product (256 walkers), scaled by walkers",
                         # V slices [Vr; Vi; -Vi] (3 x 3 M^2 bytes), A slices (3 x 2 N M), C in FP32 (8 N M)
                         "algorithmic_bytes_per_launch": W * (3.0 * 3 * spec.M * spec.M + 3.0 * 2 * spec.N * spec.M
                                                              + 4.0 * 2 * spec.N * spec.M)})
    roofline.update({"algorithmic_flops_per_launch": alg, "launch_ms": launch_ms, "launches_timed": t_n,
                     "traffic": traffic,
                     "vhs_product": {"launch_ms": v_launch, "algorithmic_flops_per_launch": v_alg,
                                     "achieved": v_alg / (v_launch * 1e-3) / 1e12 if v_launch else None,
                                     "columns": "packed upper triangle M(M+1)/2" if m["vhs_packed"] else "full M*M"}})
    tot = sum(v[0] for k, v in ph.items() if k not in ("vHS_gemm", "taylor_gemm"))
    phases = {k: {"ms_per_step": v[0] / args.steps, "share": v[0] / tot if tot else None}
              for k, v in ph.items() if v[1] > 0 and k not in ("vHS_gemm", "taylor_gemm")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_port_rate(cfg)
        cpu.pop("seconds", None)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    dtype = {"fp64": "f64", "mixed": "bf16x3 split (fp32 accumulate) + f64", "mixed-fp32":
             "bf16x6 split (fp32 accumulate) + f64", "int8x3": "int8 slices x3 (exact int32 accumulate) + f64",
             "int8x2": "int8 slices x2 (exact int32 accumulate) + f64"}[args.precision]
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": workload_config(cfg, spec, args.precision, world), "tiles": m.get("tiles"),
            "algorithmic_tflops": step_flops(spec.M, spec.N, spec.Nc) * W * args.steps * world / (ms * 1e-3) / 1e12,
            "gpu_launches": m["launches"], "clocks": m["clocks"], "e2e": e2e, "roofline": roofline,
            "fp64_comparison": compare, "phases": phases, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
