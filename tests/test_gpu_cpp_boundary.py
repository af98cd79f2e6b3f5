"""A C++ program compiled against include/safire_b200.hpp drives the GPU path through the reference's
names (det_ops::MixedDensityMatrix, HamiltonianOperations::vbias / vHS / energy /
getOneBodyPropagatorMatrix, WalkerSet, AFQMCBasePropagator) on device buffers, as a maintainer
swapping the reference's templates for this header would; its outputs are checked against the
FP64 oracle at 1e-10 (relative, max-norm), and the WalkerSet members by their definitions."""
import os
import shutil
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import afqmc_oracle as O  # noqa: E402
from safire_b200 import build, synthetic  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
W, DT, SEED = 5, 0.005, 3

PROGRAM = r'''
#include <cstdio>
#include <fstream>
#include <vector>
#include <cuda_runtime.h>
#include "safire_b200.hpp"
using namespace safire_b200;
using C = ComplexType;

template <class T> std::vector<T> load(const std::string& d, const char* n, size_t count) {
  std::vector<T> v(count);
  std::ifstream f(d + "/" + n, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * count);
  if (!f) throw std::runtime_error(std::string("read ") + n);
  return v;
}
template <class T> void save(const std::string& d, const char* n, const std::vector<T>& v) {
  std::ofstream f(d + "/" + n, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), sizeof(T) * v.size());
}
template <class T> T* dev(const std::vector<T>& h) {
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * h.size()) != cudaSuccess) throw std::runtime_error("cudaMalloc");
  cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return static_cast<T*>(p);
}
template <class T> std::vector<T> back(const T* d, size_t count) {
  std::vector<T> h(count);
  cudaMemcpy(h.data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost);
  return h;
}

int main(int argc, char** argv) {
  const std::string d = argv[1];
  const auto dims = load<int>(d, "dims", 4);
  const int M = dims[0], N = dims[1], Nc = dims[2], W = dims[3];
  const auto sc = load<double>(d, "scalars", 3);  // dt, Eshift, seed
  const double dt = sc[0];
  const auto hcore = load<double>(d, "hcore", size_t(M) * M);
  const auto Likn = load<double>(d, "Likn", size_t(M) * M * Nc);
  const auto PsiT = load<C>(d, "PsiT", size_t(N) * M);
  const auto SMh = load<C>(d, "SM", size_t(W) * M * N);
  const auto Xh = load<C>(d, "X", size_t(W) * Nc);

  // det_ops::MixedDensityMatrix / Log_Overlap on caller-owned device buffers
  C* dA = dev(PsiT);
  C* dB = dev(SMh);
  C* dG = dev(std::vector<C>(size_t(W) * N * M));
  C* dov = dev(std::vector<C>(W));
  size_t ws_bytes = det_ops::workspace_size(SFQ_OP_MIXED_DENSITY_MATRIX, W, M, N);
  void* ws = nullptr;
  cudaMalloc(&ws, ws_bytes);
  det_ops::MixedDensityMatrix(dA, dB, dG, dov, W, M, N, true, ws, ws_bytes);
  cudaFree(ws);
  save(d, "G", back(dG, size_t(W) * N * M));
  save(d, "ovlp", back(dov, W));

  // an engine (the objects execute_simulation builds) and the HamiltonianOperations view of its tensors
  sfq_engine_params_t p;
  sfq_engine_params_default(&p);
  p.nmo = M; p.nel = N; p.nchol = Nc; p.nwalk = W; p.dt = dt; p.seed = (unsigned long long)sc[2];
  Engine eng(p, hcore.data(), Likn.data(), PsiT.data());
  sfq_engine_info_t info;
  check(sfq_engine_info(eng.handle(), &info));
  HamiltonianOperations ham(M, N, Nc, static_cast<const double*>(info.Likn), info.Lnak, info.lnak_complex != 0,
                            static_cast<const C*>(info.haj), 0.0, static_cast<const double*>(info.hcore),
                            static_cast<const double*>(info.v0));
  C* dv = dev(std::vector<C>(size_t(W) * Nc));
  ham.vbias(dG, dv, W, dt);
  save(d, "vbias", back(dv, size_t(W) * Nc));
  C* dX = dev(Xh);
  C* dV = dev(std::vector<C>(size_t(W) * M * M));
  ham.vHS(dX, dV, W, dt);
  save(d, "vHS", back(dV, size_t(W) * M * M));
  C* dE = dev(std::vector<C>(size_t(W) * 3));
  size_t ews = sfq_workspace_size(SFQ_OP_ENERGY, W, M, N, Nc);
  void* ew = nullptr;
  cudaMalloc(&ew, ews);
  ham.energy(dE, dG, W, ew, ews);
  cudaFree(ew);
  save(d, "energy", back(dE, size_t(W) * 3));
  std::vector<C> vmf(Nc);
  for (int n = 0; n < Nc; ++n) vmf[n] = C(back(static_cast<const double*>(info.vmf) + n, 1)[0], 0.0);
  save(d, "H1", ham.getOneBodyPropagatorMatrix(dt, vmf));
  auto vd = ham.vHS_dims();
  std::vector<int> meta = {std::get<0>(vd), std::get<1>(vd), int(ham.getHamType() == HamiltonianType::real_dense_factorized),
                           int(ham.getFieldTypes().size()), ham.getFieldTypes()[0]};

  // WalkerSet + AFQMCBasePropagator: the engine's walkers after the energy that seeds the pseudo
  // energies (execute.cpp:172-184), two steps and an orthogonalization
  WalkerSet wset(eng);
  AFQMCBasePropagator prop(eng);
  check(sfq_engine_set_walkers(eng.handle(), SMh.data(), nullptr));
  std::vector<C> E3(size_t(W) * 3);
  check(sfq_engine_energy(eng.handle(), 1, E3.data()));
  prop.set_rng_block_size(Nc);
  prop.Propagate(wset, sc[1]);
  prop.Propagate(wset, sc[1], 0);
  prop.Orthogonalize(wset);
  save(d, "SM_prop", wset.SlaterMatrices());
  save(d, "weight", wset.getProperty(WEIGHT));
  save(d, "ovlp_prop", wset.getProperty(OVLP));
  std::vector<C> ph(W);
  for (int w = 0; w < W; ++w) ph[w] = C(0.5 + w, -0.25 * w);
  wset.setProperty(PHASE, ph);
  save(d, "phase_set", wset.getProperty(PHASE));
  wset.copy_walker(0, 2);
  save(d, "SM_copy", wset.SlaterMatrices());
  wset.resize(W + 2);
  meta.push_back(wset.size());
  save(d, "SM_resized", wset.SlaterMatrices());
  save(d, "weight_resized", wset.getProperty(WEIGHT));
  int refused = 0;
  try {
    wset.getProperty(SMN);
  } catch (const Error& e) {
    refused = e.code;
  }
  meta.push_back(refused);
  save(d, "meta", meta);
  std::printf("ok\n");
  return 0;
}
'''


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def test_cpp_program_drives_the_gpu_path_through_the_reference_names(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None or not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("no g++ or CUDA headers")
    lib = build.build()
    s = synthetic.make_system(synthetic.CFG_SMALL)
    M, N, Nc = s.M, s.N, s.Nc
    rng = np.random.default_rng(5)
    SM = s.initial_walkers(W) + 0.05 * (rng.standard_normal((W, M, N)) + 1j * rng.standard_normal((W, M, N)))
    X = rng.standard_normal((W, Nc)) + 1j * rng.standard_normal((W, Nc))
    ham = O.Hamiltonian(s.hcore, s.Likn, s.PsiT)
    # the oracle's own run from these walkers: Eshift from their energy (init_walkers)
    wo = O.Walkers(SM.copy())
    Esh = O.init_walkers(ham, wo)
    d = str(tmp_path)
    for name, arr in (("dims", np.array([M, N, Nc, W], np.int32)), ("scalars", np.array([DT, Esh, SEED], np.float64)),
                      ("hcore", s.hcore), ("Likn", s.Likn), ("PsiT", s.PsiT), ("SM", SM), ("X", X)):
        np.ascontiguousarray(arr).tofile(os.path.join(d, name))
    src = os.path.join(d, "prog.cpp")
    with open(src, "w") as f:
        f.write(PROGRAM)
    exe = os.path.join(d, "prog")
    r = subprocess.run([gxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
                        src, lib, "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-o", exe,
                        "-Wl,-rpath," + os.path.dirname(lib) + ":" + os.path.join(CUDA, "lib64")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe, d], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.stdout, out.stderr)

    def rd(name, shape, dtype=np.complex128):
        return np.fromfile(os.path.join(d, name), dtype=dtype).reshape(shape)

    Go, ovo = O.mixed_density_matrix(s.PsiT, SM)
    G = rd("G", (W, N, M))
    assert _rel(G, Go) < 1e-10
    assert _rel(rd("ovlp", (W,)), ovo) < 1e-10
    assert _rel(rd("vbias", (W, Nc)), ham.vbias(Go, DT)) < 1e-10
    assert _rel(rd("vHS", (W, M, M)), ham.vHS(X, DT)) < 1e-10
    assert _rel(rd("energy", (W, 3)), ham.energy(Go)) < 1e-10
    vmf = ham.mean_field(DT).real
    H1o = DT * (s.hcore + ham.v0) + ham.vHS(vmf[None].astype(np.complex128), DT)[0].real
    assert _rel(rd("H1", (1, M, M)).real[0], H1o) < 1e-10
    meta = rd("meta", (7,), np.int32)
    assert list(meta[:5]) == [1, 1, 1, Nc, 0]  # vHS_dims (1, 1), real dense, Nc continuous charge fields
    # two steps and an orthogonalization against the oracle on the same Philox fields
    prop = O.Propagator(ham, DT, seed=SEED)
    for st in range(2):
        prop.propagate(wo, Esh, st)
    prop.orthogonalize(wo)
    assert _rel(rd("SM_prop", (W, M, N)), wo.SM) < 1e-10
    assert _rel(rd("weight", (W,)), wo.weight) < 1e-10
    assert _rel(rd("ovlp_prop", (W,)), wo.ovlp) < 1e-10
    ph = np.array([complex(0.5 + w, -0.25 * w) for w in range(W)])
    assert np.array_equal(rd("phase_set", (W,)), ph)
    Sc = rd("SM_copy", (W, M, N))
    Sp = rd("SM_prop", (W, M, N))
    assert np.array_equal(Sc[2], Sc[0]) and np.array_equal(Sc[[0, 1, 3, 4]], Sp[[0, 1, 3, 4]])
    assert meta[5] == W + 2  # resize: slots W, W+1 filled from 0, 1 (round robin)
    Sr = rd("SM_resized", (W + 2, M, N))
    assert np.array_equal(Sr[:W], Sc) and np.array_equal(Sr[W:], Sc[:2])
    wr = rd("weight_resized", (W + 2,))
    assert np.array_equal(wr[W:], wr[:2])
    assert meta[6] == 2  # SMN is not a property column: SFQ_ERR_ARG
