"""Seeded synthetic dense-Cholesky systems (stand-in for the reference's HDF5 inputs).

The reference reads ``Hamiltonian/hcore`` and ``Hamiltonian/DenseFactorized/L`` from HDF5
(src/AFQMC/Hamiltonians/RealDenseHamiltonian.cpp:87-134) and the trial from
``Wavefunction/NOMSD/PsiT_*`` (src/AFQMC/Utilities/readWfn.cpp:50-131).  No HDF5 stack is
available here, so systems are generated in memory with the distributions below:

* hcore: real symmetric, diagonal -2 + 0.25 i, off-diagonal N(0, 0.05^2);
* Nc real symmetric Cholesky vectors L_n (M x M), upper-triangle entries N(0,1) mirrored,
  scaled by exp(-n / decay) / sqrt(M); stored as Likn[i, k, n] (n fastest), the reference's
  layout (Real3IndexFactorization.hpp:668);
* RHF trial: the lowest N eigenvectors of hcore, PsiT = Psi^T (N x M);
* walkers start as copies of the trial (M x N).

All draws use numpy's Philox bit generator from the system seed, so every process (oracle,
GPU path, CPU baseline) sees identical arrays.
"""
import math
from dataclasses import dataclass

import numpy as np


@dataclass
class SystemSpec:
    M: int
    N: int
    Nc: int
    decay: float
    seed: int = 0

    @property
    def name(self):
        return f"M{self.M}_N{self.N}_Nc{self.Nc}"


# The three single-system configurations the benchmark and tests use.
CFG_SMALL = SystemSpec(M=24, N=6, Nc=96, decay=24.0)        # CPU-runnable case
CFG_MEDIUM = SystemSpec(M=128, N=32, Nc=640, decay=128.0)    # FP64 drop-in case
CFG_LARGE = SystemSpec(M=400, N=100, Nc=2400, decay=400.0)   # precision / headline case


@dataclass
class System:
    spec: SystemSpec
    hcore: np.ndarray      # (M, M) float64
    Likn: np.ndarray       # (M, M, Nc) float64
    PsiT: np.ndarray       # (N, M) complex128; COLLINEAR: the up rows over the down rows
    E0: float = 0.0
    nel_dn: int = -1       # COLLINEAR walkers: the last nel_dn rows of PsiT are the down spin; -1: CLOSED
    npol: int = 1          # 2: NONCOLLINEAR walkers, PsiT (N, 2M) spinor orbitals
    ci: np.ndarray = None  # multi-determinant trial: the coefficients, PsiT then (ndet, N, M or 2M)

    @property
    def M(self):
        return self.spec.M

    @property
    def N(self):
        return self.spec.N

    @property
    def Nc(self):
        return self.spec.Nc

    def initial_walkers(self, nwalk):
        psi = np.conj(self.PsiT.T)
        return np.ascontiguousarray(np.broadcast_to(psi, (nwalk,) + psi.shape)).astype(np.complex128)


def make_system(spec: SystemSpec) -> System:
    M, N, Nc = spec.M, spec.N, spec.Nc
    rng = np.random.Generator(np.random.Philox(spec.seed))
    h = rng.normal(0.0, 0.05, size=(M, M))
    h = np.triu(h, 1)
    h = h + h.T
    h[np.diag_indices(M)] = -2.0 + 0.25 * np.arange(M)
    L = np.empty((M, M, Nc), dtype=np.float64)
    scale = np.exp(-np.arange(Nc) / spec.decay) / math.sqrt(M)
    iu = np.triu_indices(M)
    blk = max(1, min(Nc, 64))
    for n0 in range(0, Nc, blk):
        n1 = min(Nc, n0 + blk)
        A = rng.standard_normal(size=(n1 - n0, iu[0].size))
        S = np.zeros((n1 - n0, M, M))
        S[:, iu[0], iu[1]] = A
        S = S + np.transpose(np.triu(S, 1), (0, 2, 1))
        S *= scale[n0:n1, None, None]
        L[:, :, n0:n1] = np.transpose(S, (1, 2, 0))
    evals, evecs = np.linalg.eigh(h)
    psi = evecs[:, :N]
    PsiT = np.ascontiguousarray(psi.T).astype(np.complex128)
    return System(spec=spec, hcore=h, Likn=L, PsiT=PsiT, E0=0.0)
