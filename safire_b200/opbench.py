"""Time one AFQMC operation in isolation (CUDA events), e.g. for profiling a single kernel.

  python -m safire_b200.opbench --op vhs --M 400 --N 100 --Nc 2400 --W 64 --reps 3

Operands are random with the shapes of the path; prints one JSON line per op with the
average device time per call and the algorithmic TFLOP/s.  `mixed_step` runs whole propagation
steps of a resident mixed-precision engine on a synthetic system of the given sizes (the Taylor
and P1 products do not depend on Nc, so a small Nc profiles them in a small footprint).
"""
import argparse
import json

import numpy as np
import torch

from . import afqmc


def _flops(op, M, N, Nc, W):
    return {
        "vhs": 4.0 * M * M * Nc * W,
        "vbias": 8.0 * N * M * Nc * W,
        "propagate": 64.0 * M * M * N * W,
        "density": (8.0 * N * N * M + 8.0 * N * N * M + 8.0 * N ** 3) * W,
        "inverse": 8.0 * N ** 3 * W,
        "energy": 8.0 * N * N * M * Nc * W,
        "orthogonalize": 2 * (8.0 * N * N * M * 2) * W,
        "umma_vhs": 2.0 * (2 * W) * M * M * Nc,   # one real product of the split GEMM
        "umma_planes": 2.0 * (2 * W) * M * M * Nc,
        "mixed_step": (8.0 * N * M * Nc + 4.0 * M * M * Nc + 64.0 * M * M * N + 24.0 * N * N * M
                       + (32.0 / 3.0) * N ** 3) * W,
    }[op]


def _mixed_step(M, N, Nc, W, reps, warm):
    from . import capi, synthetic
    s = synthetic.make_system(synthetic.SystemSpec(M=M, N=N, Nc=Nc, decay=max(Nc / 6.0, 1.0), seed=0))
    eng = afqmc.AfqmcEngine(s, W, dt=0.0005, seed=1, precision=capi.PRECISION_MIXED)
    Esh = eng.init()
    ext = torch.cuda.ExternalStream(eng.stream)
    step = 0
    for _ in range(warm):
        eng.propagate(Esh, step)
        step += 1
    eng.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(reps):
        eng.propagate(Esh, step)
        step += 1
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    eng.close()
    return ms


def run(op, M, N, Nc, W, reps, warm=2, real_lnak=True):
    if op == "mixed_step":
        ms = _mixed_step(M, N, Nc, W, reps, warm)
        fl = _flops(op, M, N, Nc, W)
        return {"op": op, "M": M, "N": N, "Nc": Nc, "W": W, "ms": ms, "tflops": fl / (ms * 1e-3) / 1e12}
    g = torch.Generator(device="cuda").manual_seed(0)

    def crand(*shape):
        return torch.complex(torch.randn(*shape, generator=g, device="cuda", dtype=torch.float64),
                             torch.randn(*shape, generator=g, device="cuda", dtype=torch.float64))

    if op == "vhs":
        L = torch.randn(M, M, Nc, generator=g, device="cuda", dtype=torch.float64)
        X = crand(W, Nc)
        fn = lambda: afqmc.vHS(L, X, 0.005)  # noqa: E731
    elif op == "vbias":
        G = crand(W, N, M)
        Ln = torch.randn(Nc, N, M, generator=g, device="cuda", dtype=torch.float64) if real_lnak else crand(Nc, N, M)
        fn = lambda: afqmc.vbias(G, Ln, 0.005)  # noqa: E731
    elif op == "propagate":
        SM = crand(W, M, N)
        P1 = torch.eye(M, device="cuda", dtype=torch.float64)
        V = crand(W, M, M) * 1e-3
        fn = lambda: afqmc.Propagate(SM, P1, V, 6)  # noqa: E731
    elif op == "density":
        A = torch.randn(N, M, generator=g, device="cuda", dtype=torch.float64)
        B = crand(W, M, N)
        fn = lambda: afqmc.MixedDensityMatrix(A, B)  # noqa: E731
    elif op == "inverse":
        # the per-walker overlap matrices' inverse and log det (Gauss-Jordan), N x N
        A = crand(W, N, N) + 4.0 * torch.eye(N, dtype=torch.complex128, device="cuda")
        fn = lambda: afqmc.inverse_logdet(A)  # noqa: E731
    elif op == "energy":
        G = crand(W, N, M) * 0.01
        haj = crand(N, M)
        Ln = torch.randn(Nc, N, M, generator=g, device="cuda", dtype=torch.float64)
        fn = lambda: afqmc.energy(G, haj, Ln)  # noqa: E731
    elif op == "umma_vhs":
        # the vHS-shaped split-BF16 tensor-core GEMM: (2W x Nc) x (M^2 x Nc)^T, 3 products
        import ctypes
        from . import capi
        A = torch.randn(2 * W, Nc, generator=g, device="cuda", dtype=torch.float64)
        B = torch.randn(M * M, Nc, generator=g, device="cuda", dtype=torch.float64)
        C = torch.empty(2 * W, M * M, device="cuda", dtype=torch.float32)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        fn = lambda: capi.check(capi.lib().sfq_gemm_split_bf16(A.data_ptr(), B.data_ptr(), C.data_ptr(), 2 * W,  # noqa
                                                               M * M, Nc, 1, 0, 0, 3, 0, st))
    elif op == "umma_planes":
        # the same GEMM on pre-split planes: tensor-core time only
        import ctypes
        from . import capi
        L = capi.lib()
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        A = torch.randn(2 * W, Nc, generator=g, device="cuda", dtype=torch.float64)
        B = torch.randn(M * M, Nc, generator=g, device="cuda", dtype=torch.float64)
        env = __import__("os").environ
        npl = int(env.get("SFQ_PLANES", "2"))
        tn = int(env.get("SFQ_TILE_N", "0"))
        pa = [torch.empty(A.numel(), dtype=torch.bfloat16, device="cuda") for _ in range(npl)]
        pb = [torch.empty(B.numel(), dtype=torch.bfloat16, device="cuda") for _ in range(npl)]
        ptr3 = lambda ps: [ps[q].data_ptr() if q < len(ps) else None for q in range(3)]  # noqa: E731
        capi.check(L.sfq_split_bf16(A.data_ptr(), A.numel(), *ptr3(pa), st))
        capi.check(L.sfq_split_bf16(B.data_ptr(), B.numel(), *ptr3(pb), st))
        del B
        C = torch.empty(2 * W, M * M, device="cuda", dtype=torch.float32)
        VP3 = ctypes.c_void_p * 3
        Aarr, Barr = VP3(*ptr3(pa)), VP3(*ptr3(pb))
        fn = lambda: capi.check(L.sfq_gemm_bf16_planes(Aarr, Barr, npl, C.data_ptr(), 2 * W, M * M, Nc, 1,  # noqa
                                                       0, 0, 1.0, 0.0, tn, st))
    elif op == "orthogonalize":
        SM = crand(W, M, N)
        fn = lambda: afqmc.orthogonalize(SM)  # noqa: E731
    else:
        raise ValueError(op)
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    fl = _flops(op, M, N, Nc, W)
    return {"op": op, "M": M, "N": N, "Nc": Nc, "W": W, "ms": ms, "tflops": fl / (ms * 1e-3) / 1e12}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", default="vhs")
    ap.add_argument("--M", type=int, default=400)
    ap.add_argument("--N", type=int, default=100)
    ap.add_argument("--Nc", type=int, default=2400)
    ap.add_argument("--W", type=int, default=64)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warm", type=int, default=2)
    a = ap.parse_args()
    for op in a.op.split(","):
        print(json.dumps(run(op, a.M, a.N, a.Nc, a.W, a.reps, a.warm)), flush=True)


if __name__ == "__main__":
    main()
