"""ORACLE (test infrastructure only) -- FP64 CPU restatement of SAFIRE's AFQMC hot path.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module, and only as the checker / the timed CPU baseline; the product path (safire_b200)
never calls it.

It restates, function by function, the reference's CLOSED-shell, single-determinant,
dense-real-Cholesky path (paths relative to the SAFIRE source tree):

  log_determinant_from_getrf    src/numerics/operations/determinants_impl.hpp:33-75
  log_determinant_from_geqrf    src/numerics/operations/determinants_impl.hpp:78-108
  log_overlap_impl              src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp:120-156
  getri_or_zero                 src/numerics/nda_functions.hpp:422-438
  inverse_logdet                src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp:42-76
  MixedDensityMatrix            src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp:544-601
  Log_Overlap                   src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp:437-447
  NOMSD::Log_Overlap (CLOSED x2) src/AFQMC/Wavefunctions/NOMSD.cpp:280-300
  NOMSD::DensityMatrix          src/AFQMC/Wavefunctions/NOMSD.hpp:293-343
  Real3IndexFactorization       src/AFQMC/HamiltonianOperations/Real3IndexFactorization.hpp
      vHS :282-326, vbias :328-428, energy :138-174, energy_impl :476-590,
      getOneBodyPropagatorMatrix :99-124
  add_one_body_shifts           src/AFQMC/HamiltonianOperations/detail/one_body.hpp:65-85
  half rotation, v0             src/AFQMC/Hamiltonians/RealDenseHamiltonian.cpp:138-180
  NOMSD::vMF                    src/AFQMC/Wavefunctions/NOMSD.cpp:437-466
  generateP1 / exp_hermitian    src/AFQMC/Propagators/AFQMCBasePropagator.cpp:43-214;
                                src/numerics/operations/exp.hpp:28-60
  assemble_X / construct_X      src/AFQMC/Propagators/AFQMCBasePropagator.cpp:687-733;
                                src/AFQMC/Propagators/construct_X_kernel.hpp:34-87
  probit (Acklam)               src/AFQMC/Utilities/probit.h:58-136
  Propagate (step 1..7)         src/AFQMC/Propagators/AFQMCBasePropagator.cpp:290-392
  apply_expM / propagate_impl   src/AFQMC/SlaterDeterminantOperations/propagate.hpp:45-70,247-298
  walker_update / bounds        src/AFQMC/Propagators/WalkerSetUpdate.hpp:46-218
  orthogonalize                 src/AFQMC/SlaterDeterminantOperations/orthogonalize.hpp:135-169
  comb / swap_walkers_async     src/AFQMC/Walkers/population_control.hpp:34-65,143-255
  plan_walker_exchange / moves  src/AFQMC/Walkers/population_control.hpp:73-209 (sharded walkers)
  averagePseudoEnergy / averageEnergy   src/AFQMC/Drivers/average_energy.hpp:33-76
  EnergyEstimator::measure      src/AFQMC/Estimators/EnergyEstimator.h:51-100
  run_afqmc step loop           src/AFQMC/Drivers/run_afqmc.cpp:69-113

Beyond the CLOSED single-determinant path, restated the same way and pinned the same way (below):
  CollinearHamiltonian          the COLLINEAR branches of NOMSD / Real3IndexFactorization (per spin)
  NoncollinearHamiltonian       the npol = 2 branches (spinor walkers, polarization-independent H)
  MultiDetHamiltonian           NOMSD with ndet > 1 (NOMSD.cpp:159-331,466-512)
  measure_mixed_rdms            MixedEstimator + OneRDM / DiagonalTwoRDM (MixedEstimator.hpp:37-147)
  BackPropEstimator             BackPropEstimator + BackPropagate (BackPropEstimator.hpp:36-275,
                                AFQMCBasePropagator.cpp:404-526)
  run_seeded, rebinned_average  execute_simulation + run_afqmc on the reference's host streams
                                (oracle.mt19937); safiretools' Results.average

LAPACK arithmetic at the boundary (the reference reaches it through TRIQS/nda @5046352):
zgetrf / zgetri / zgeqrf / zungqr from scipy's OpenBLAS, and numpy's eigh (zheevd).

Auxiliary fields come from ``oracle.philox`` (Philox-4x32-10, stream 1); the comb draws from
stream 0.  The reference uses mt19937 here (src/utilities/Random.hpp:37-51); the injection
point ``sampleUniformFields`` is the same.  ``run_seeded`` replays a whole stage on the reference's
own streams (``oracle.mt19937``) and reproduces the reference's recorded seeded BH run
(tests/functional/snapshot_references/BH/dense_rhf_basis_closed/rhf_nomsd/closed) to ~1e-14.
"""
import math

import numpy as np
import scipy.linalg.lapack as lapack

from . import philox

SMALL = np.finfo(np.float64).tiny  # numeric_limits<double>::min(), determinants_impl.hpp:40


# --------------------------------------------------------------------------------------------
# log det, LU, inverse (determinants_impl.hpp:33-75; nda_functions.hpp:422-438)
# --------------------------------------------------------------------------------------------
def log_det_from_getrf(lu, piv, res=0j):
    """Sum_i log(+-U_ii + tiny), pivot sign per row swap, imag folded into [-pi, pi].

    ``piv`` is LAPACK's 0-based pivot vector (scipy), so "no swap" is piv[i] == i; the
    reference compares the 1-based ipiv to i+1 (determinants_impl.hpp:46-50).  ``res``
    accumulates, as in the reference.
    """
    n = lu.shape[0]
    for i in range(n):
        d = complex(lu[i, i])
        if piv[i] == i:
            res += np.log(d + SMALL)
        else:
            res += np.log(-d + SMALL)
    im = res.imag
    if im > math.pi:
        while im > math.pi:
            im -= 2 * math.pi
    elif im < -math.pi:
        while im < -math.pi:
            im += 2 * math.pi
    return complex(res.real, im)


def lu_logdet_inverse(T, res=0j, invert=True):
    """getrf + log det + getri_or_zero for one N x N complex matrix."""
    lu, piv, info = lapack.zgetrf(np.asarray(T, dtype=np.complex128))
    ld = log_det_from_getrf(lu, piv, res)
    if not invert:
        return ld, None
    inv, info2 = lapack.zgetri(lu, piv)
    if info2 != 0:
        inv = np.zeros_like(inv)
    return ld, inv


def inverse_logdet(A):
    """density_matrix.hpp:82-108 -- batched (nbatch, N, N): returns (inverse, logdet)."""
    A = np.asarray(A, dtype=np.complex128)
    inv = np.empty_like(A)
    ld = np.zeros(A.shape[0], dtype=np.complex128)
    for b in range(A.shape[0]):
        ld[b], inv[b] = lu_logdet_inverse(A[b])
    return inv, ld


# --------------------------------------------------------------------------------------------
# Overlaps and mixed density matrix (density_matrix.hpp:120-156,437-447,544-601)
# --------------------------------------------------------------------------------------------
def mixed_density_matrix(A, B, compact=True, ovlp=None):
    """A = PsiT (N x M, herm=true form), B = walkers (W, M, N).

    Returns (G, ovlp) with G (W, N, M) when compact (G = T(T^-1) * T(B)), or (W, M, M)
    otherwise (G = conj-free A^T * T^-T * B^T, density_matrix.hpp:580-585).
    ``ovlp`` accumulates (log_determinant_from_getrf adds to res).
    """
    A = np.asarray(A, dtype=np.complex128)
    B = np.asarray(B, dtype=np.complex128)
    W, M, N = B.shape
    if ovlp is None:
        ovlp = np.zeros(W, dtype=np.complex128)
    else:
        ovlp = np.array(ovlp, dtype=np.complex128)
    if N == 0:
        return np.zeros((W, 0, M) if compact else (W, M, M), np.complex128), ovlp
    T = A @ B                                   # (W, N, N)   math::product(A,B,TNN)
    Tinv = np.empty_like(T)
    for w in range(W):
        ovlp[w], Tinv[w] = lu_logdet_inverse(T[w], ovlp[w])
    # C = T(TNN) * T(B)  -> C[w] = Tinv[w]^T @ B[w]^T
    Gc = np.transpose(Tinv, (0, 2, 1)) @ np.transpose(B, (0, 2, 1))   # (W, N, M)
    if compact:
        return Gc, ovlp
    # herm: C = T(A) * T2 with T2 = T(TNN) * T(B)
    return A.T[None, :, :] @ Gc, ovlp


def log_overlap(A, B, ovlp=None):
    """det_ops::Log_Overlap (density_matrix.hpp:437-447): accumulating, no inverse."""
    A = np.asarray(A, dtype=np.complex128)
    B = np.asarray(B, dtype=np.complex128)
    W = B.shape[0]
    ovlp = np.zeros(W, np.complex128) if ovlp is None else np.array(ovlp, np.complex128)
    if B.shape[2] == 0:
        return ovlp
    T = A @ B
    for w in range(W):
        ovlp[w], _ = lu_logdet_inverse(T[w], ovlp[w], invert=False)
    return ovlp


def log_overlap_closed(PsiT, Wk):
    """NOMSD::Log_Overlap, ndet = 1, CLOSED: 2 * Log_Overlap + log(conj(ci0)), ci0 = 1."""
    return 2.0 * log_overlap(PsiT, Wk) + np.log(np.conj(1.0 + 0j))


# --------------------------------------------------------------------------------------------
# Hamiltonian setup (RealDenseHamiltonian.cpp:138-180; one_body.hpp:65-153)
# --------------------------------------------------------------------------------------------
class Hamiltonian:
    """Dense real Cholesky Hamiltonian + single-determinant CLOSED trial.

    hcore (M, M) real symmetric; Likn (M, M, Nc) real, L[i, k, n]; PsiT (N, M) complex.
    """

    def __init__(self, hcore, Likn, PsiT, E0=0.0):
        self.hcore = np.asarray(hcore, dtype=np.float64)
        self.Likn = np.ascontiguousarray(Likn, dtype=np.float64)
        self.PsiT = np.asarray(PsiT, dtype=np.complex128)
        self.E0 = float(E0)
        self.M = self.hcore.shape[0]
        self.N = self.PsiT.shape[0]
        self.Nc = self.Likn.shape[2]
        M, N, Nc = self.M, self.N, self.Nc
        # haj = PsiT * hcore (one_body.hpp:124-153)
        self.haj = self.PsiT @ self.hcore.astype(np.complex128)
        # Lnak[n, a, k] = sum_i PsiT[a, i] L[i, k, n]  (RealDenseHamiltonian.cpp:141-161)
        L2 = self.Likn.reshape(M, M * Nc)
        Lak_n = (self.PsiT.real @ L2 + 1j * (self.PsiT.imag @ L2)).reshape(N, M, Nc)
        self.Lnak = np.ascontiguousarray(np.transpose(Lak_n, (2, 0, 1)))
        # v0[i, l] = -0.5 sum_{j,n} L[i, j, n] L[l, j, n]  (RealDenseHamiltonian.cpp:165-180)
        Lf = self.Likn.reshape(M, M * Nc)
        self.v0 = -0.5 * (Lf @ Lf.T)

    # Real3IndexFactorization::vbias, CLOSED, ndet = 1 (:328-428): a = 2 sqrt(dt)
    def vbias(self, G, dt):
        W = G.shape[0]
        a = 2.0 * math.sqrt(dt)
        G2 = G.reshape(W, self.N * self.M)
        L2 = self.Lnak.reshape(self.Nc, self.N * self.M)
        return a * (G2 @ L2.T)

    # Real3IndexFactorization::vHS (:282-326): v[w, i, k] = sqrt(dt) sum_n L[i, k, n] X[w, n]
    def vHS(self, X, dt):
        W = X.shape[0]
        a = math.sqrt(dt)
        L2 = self.Likn.reshape(self.M * self.M, self.Nc)
        Xr = np.ascontiguousarray(X.real.T)
        Xi = np.ascontiguousarray(X.imag.T)
        v = (L2 @ Xr) + 1j * (L2 @ Xi)            # (M*M, W)
        return a * np.ascontiguousarray(v.T).reshape(W, self.M, self.M)

    # Real3IndexFactorization::energy / energy_impl, CLOSED (:138-174, :476-590)
    def energy(self, G, addH1=True, addEJ=True, addEXX=True, chunk=None):
        W = G.shape[0]
        N, M, Nc = self.N, self.M, self.Nc
        scl = 2.0
        E = np.zeros((W, 3), dtype=np.complex128)
        if addH1:
            E[:, 0] = self.E0
            E[:, 0] += scl * np.einsum('waj,aj->w', G, self.haj)
        Kl = np.zeros((W, Nc), dtype=np.complex128)
        if addEXX:
            if chunk is None:
                chunk = max(1, min(Nc, int(2e8 // max(1, W * N * N))))
            L3 = self.Lnak
            for n0 in range(0, Nc, chunk):
                n1 = min(Nc, n0 + chunk)
                Lc = L3[n0:n1].reshape((n1 - n0) * N, M)          # rows (n, a)
                T = (G.reshape(W * N, M) @ Lc.T).reshape(W, N, n1 - n0, N)  # T[w,b,n,a]
                # E1 += -0.5 scl sum_abn T[w,a,n,b] T[w,b,n,a]
                E[:, 1] += -0.5 * scl * np.einsum('wanb,wbna->w', T, T)
                if addEJ:
                    Kl[:, n0:n1] += np.einsum('wana->wn', T)
        if addEJ:
            E[:, 2] += 0.5 * 4.0 * np.einsum('wn,wn->w', Kl, Kl)
        return E

    # Real3IndexFactorization::getOneBodyPropagatorMatrix (:99-124) + add_one_body_shifts
    def one_body_propagator_matrix(self, dt, vMF):
        shift = self.vHS(np.asarray(vMF, np.complex128)[None, :], dt)[0]
        return dt * self.hcore + dt * self.v0 + shift

    # the walker type's view of the NOMSD trial (NOMSD.hpp:293-343, NOMSD.cpp:280-300): CLOSED walkers
    # are one (M, N) Slater matrix, the overlap counts it twice
    def green(self, SM):
        G, ov = mixed_density_matrix(self.PsiT, SM, compact=True)
        return G, 2.0 * ov

    def log_overlap(self, SM):
        return log_overlap_closed(self.PsiT, SM)

    def trial_walker(self):
        return np.conj(self.PsiT.T)

    def orthogonalize(self, SM):
        return orthogonalize(SM)[0]

    def propagate(self, SM, P1, V, order):
        return propagate(SM, P1, V, order)

    def orthogonalize_ldet(self, SM):
        """det_ops::orthogonalize(wset, ldet): the walkers' QR and the log det of R."""
        return orthogonalize(SM)

    def bp_full_green(self, A, SM):
        """Full G (W, nspin, Mr, Mr) and log overlap between per-walker references A (W, n, Mr) in
        the herm form and the walkers (the batched det_ops with T = Refs^H B, density_matrix.hpp:158-195)."""
        G, ov = _batched_full_green(A, SM)
        return G[:, None], ov

    def local_energy(self, SM):
        """NOMSD::Energy(wset, E, Ov), ndet = 1: (E (W, 3), log overlaps)."""
        G, ov = self.green(SM)
        return self.energy(G), ov

    def mean_field(self, dt):
        """NOMSD::vMF, ndet = 1 (NOMSD.cpp:437-456): vbias of the trial's own G, real part kept."""
        return self.vbias(self.green(self.trial_walker()[None])[0], dt)[0].real.astype(np.complex128)

    # the pieces a multi-determinant trial combines (NOMSD.cpp:184-216,238-278,300-331)
    nspin_blocks = 1           # full-G blocks: CLOSED 1, COLLINEAR 2 spins
    vbias_scale = 2.0          # CLOSED: 2 sqrt(dt)
    ov_factor = 2.0            # DensityMatrix / Log_Overlap count a CLOSED determinant twice

    def det_log_overlap(self, SM):
        """The determinant's log overlap without the ci term (CLOSED: twice one spin's)."""
        return 2.0 * log_overlap(self.PsiT, SM)

    def full_green(self, SM):
        """det_ops::MixedDensityMatrix(compact = false) per spin: (W, nspin_blocks, Mr, Mr) and the
        accumulated log overlap as det_ops returns it (CLOSED: one spin's, not doubled)."""
        G, ov = mixed_density_matrix(self.PsiT, SM, compact=False)
        return G[:, None], ov

    def full_green_vbias(self, Gf, dt):
        """Real3IndexFactorization::vbias on a full G (:392-426): sum_s sum_ik L[i,k,n] G[w,s,i,k]."""
        W = Gf.shape[0]
        L2 = self.Likn.reshape(self.M * self.M, self.Nc)
        g = Gf.sum(axis=1).reshape(W, self.M * self.M)
        return self.vbias_scale * math.sqrt(dt) * (g @ L2)


class CollinearHamiltonian(Hamiltonian):
    """The same dense Hamiltonian for COLLINEAR walkers and a single-determinant NOMSD trial with
    PsiT_up (nup, M) and PsiT_dn (ndn, M).  A walker is one (M, nup + ndn) matrix, the up columns
    first (the reference keeps the two blocks one after the other, WalkerSetBase.h:256-264).

      half rotation   haj = [PsiT_up; PsiT_dn] hcore, Lnak per spin (RealDenseHamiltonian.cpp:141-161)
      G, overlap      MixedDensityMatrix per spin into the rows of one compact G, the overlaps
                      accumulated (NOMSD.hpp:293-343); + log(conj(ci)) (NOMSD.cpp:174-177)
      vbias           a = sqrt(dt), the two spins' G Lnak^T summed (Real3IndexFactorization.hpp:328-390)
      energy          E1 and exchange per spin with scl = 1, Coulomb 0.5 (Kl_up + Kl_dn)^2 (:138-174, :476-590)
      P1, vHS         one for both spins: the Hamiltonian is spin-independent (AFQMCBasePropagator.cpp:128-160)
      orthogonalize   each spin block on its own (orthogonalize.hpp:135-169)
    """

    def __init__(self, hcore, Likn, PsiT_up, PsiT_dn, E0=0.0, ci=1.0):
        super().__init__(hcore, Likn, PsiT_up, E0)
        self.PsiT_up = np.asarray(PsiT_up, dtype=np.complex128)
        self.PsiT_dn = np.asarray(PsiT_dn, dtype=np.complex128)
        self.nup, self.ndn = self.PsiT_up.shape[0], self.PsiT_dn.shape[0]
        self.ci = complex(ci)
        M, Nc = self.M, self.Nc
        self.N = self.nup + self.ndn
        self.haj = np.concatenate([self.PsiT_up, self.PsiT_dn]) @ self.hcore.astype(np.complex128)
        L2 = self.Likn.reshape(M, M * Nc)
        self.Lnak_s = []
        for P in (self.PsiT_up, self.PsiT_dn):
            Lak_n = (P.real @ L2 + 1j * (P.imag @ L2)).reshape(P.shape[0], M, Nc)
            self.Lnak_s.append(np.ascontiguousarray(np.transpose(Lak_n, (2, 0, 1))))
        self.Lnak = np.concatenate(self.Lnak_s, axis=1)   # (Nc, nup + ndn, M)

    def _lci(self):
        return np.log(1e-12 if abs(self.ci) < 1e-12 else np.conj(self.ci))

    def green(self, SM):
        G_up, ov = mixed_density_matrix(self.PsiT_up, SM[:, :, :self.nup], compact=True)
        G_dn, ov = mixed_density_matrix(self.PsiT_dn, SM[:, :, self.nup:], compact=True, ovlp=ov)
        return np.concatenate([G_up, G_dn], axis=1), ov + self._lci()

    def log_overlap(self, SM):
        ov = log_overlap(self.PsiT_up, SM[:, :, :self.nup])
        return log_overlap(self.PsiT_dn, SM[:, :, self.nup:], ovlp=ov) + self._lci()

    def trial_walker(self):
        return np.concatenate([np.conj(self.PsiT_up.T), np.conj(self.PsiT_dn.T)], axis=1)

    nspin_blocks = 2
    vbias_scale = 1.0
    ov_factor = 1.0

    def det_log_overlap(self, SM):
        ov = log_overlap(self.PsiT_up, SM[:, :, :self.nup])
        return log_overlap(self.PsiT_dn, SM[:, :, self.nup:], ovlp=ov)

    def full_green(self, SM):
        G_up, ov = mixed_density_matrix(self.PsiT_up, SM[:, :, :self.nup], compact=False)
        G_dn, ov = mixed_density_matrix(self.PsiT_dn, SM[:, :, self.nup:], compact=False, ovlp=ov)
        return np.stack([G_up, G_dn], axis=1), ov

    def orthogonalize_ldet(self, SM):
        up, ld = orthogonalize(SM[:, :, :self.nup])
        if self.ndn:
            dn, l2 = orthogonalize(SM[:, :, self.nup:])
            ld = ld + l2
        else:
            dn = SM[:, :, self.nup:]
        return np.concatenate([up, dn], axis=2), ld

    def bp_full_green(self, A, SM):
        Gu, ov = _batched_full_green(A[:, :self.nup], SM[:, :, :self.nup])
        Gd, o2 = _batched_full_green(A[:, self.nup:], SM[:, :, self.nup:])
        return np.stack([Gu, Gd], axis=1), ov + o2

    def orthogonalize(self, SM):
        up = orthogonalize(SM[:, :, :self.nup])[0]
        dn = orthogonalize(SM[:, :, self.nup:])[0] if self.ndn else SM[:, :, self.nup:]
        return np.concatenate([up, dn], axis=2)

    def vbias(self, G, dt):
        W = G.shape[0]
        a = math.sqrt(dt)
        v = np.zeros((W, self.Nc), np.complex128)
        rows = ((0, self.nup), (self.nup, self.N))
        for s, (r0, r1) in enumerate(rows):
            if r1 > r0:
                v += G[:, r0:r1, :].reshape(W, -1) @ self.Lnak_s[s].reshape(self.Nc, -1).T
        return a * v

    def energy(self, G, addH1=True, addEJ=True, addEXX=True, chunk=None):
        W = G.shape[0]
        M, Nc = self.M, self.Nc
        E = np.zeros((W, 3), dtype=np.complex128)
        Kl = np.zeros((W, Nc), dtype=np.complex128)
        if addH1:
            E[:, 0] = self.E0
        for s, (r0, r1) in enumerate(((0, self.nup), (self.nup, self.N))):
            n = r1 - r0
            if n == 0:
                continue
            Gs = G[:, r0:r1, :]
            if addH1:
                E[:, 0] += np.einsum('waj,aj->w', Gs, self.haj[r0:r1])
            if addEXX:
                Lc = self.Lnak_s[s].reshape(Nc * n, M)
                T = (Gs.reshape(W * n, M) @ Lc.T).reshape(W, n, Nc, n)   # T[w,b,n,a]
                E[:, 1] += -0.5 * np.einsum('wanb,wbna->w', T, T)
                if addEJ:
                    Kl += np.einsum('wana->wn', T)
        if addEJ:
            E[:, 2] += 0.5 * np.einsum('wn,wn->w', Kl, Kl)
        return E


class NoncollinearHamiltonian(Hamiltonian):
    """The same dense, spin-independent Hamiltonian for NONCOLLINEAR walkers: a walker is one
    (2M, N) spinor matrix (the two components' rows one after the other), the trial PsiT (N, 2M).

      half rotation   haj = PsiT blockdiag(hcore, hcore); Lnak[n, a, p M + k] = sum_i PsiT[a, p M + i]
                      L[i, k, n] (RealDenseHamiltonian.cpp:141-161 with npol = 2)
      G, overlap      one determinant of the 2M x N matrix, counted once (NOMSD.hpp:293-343)
      vbias           a = sqrt(dt), G Lnak^T over (a, p, k) (Real3IndexFactorization.hpp:328-390)
      energy          scale 1, the exchange tensor summed over both components (:476-560)
      P1, vHS         polarization independent: the M x M propagators act on each component
                      (getOneBodyPropagatorMatrix :99-124, propagate_impl propagate.hpp:247-298)
    """

    def __init__(self, hcore, Likn, PsiT, E0=0.0, ci=1.0):
        PsiT = np.asarray(PsiT, dtype=np.complex128)
        M = np.asarray(hcore).shape[0]
        assert PsiT.shape[1] == 2 * M
        super().__init__(hcore, Likn, PsiT[:, :M], E0)
        self.PsiT = PsiT
        self.ci = complex(ci)
        self.N = PsiT.shape[0]
        Nc = self.Nc
        h = self.hcore.astype(np.complex128)
        self.haj = np.concatenate([PsiT[:, :M] @ h, PsiT[:, M:] @ h], axis=1)
        L2 = self.Likn.reshape(M, M * Nc)
        parts = []
        for q in (PsiT[:, :M], PsiT[:, M:]):
            parts.append((q.real @ L2 + 1j * (q.imag @ L2)).reshape(self.N, M, Nc))
        self.Lnak = np.ascontiguousarray(np.transpose(np.concatenate(parts, axis=1), (2, 0, 1)))  # (Nc, N, 2M)

    def _lci(self):
        return np.log(1e-12 if abs(self.ci) < 1e-12 else np.conj(self.ci))

    def green(self, SM):
        G, ov = mixed_density_matrix(self.PsiT, SM, compact=True)
        return G, ov + self._lci()

    def log_overlap(self, SM):
        return log_overlap(self.PsiT, SM) + self._lci()

    def trial_walker(self):
        return np.conj(self.PsiT.T)

    vbias_scale = 1.0
    ov_factor = 1.0

    def det_log_overlap(self, SM):
        return log_overlap(self.PsiT, SM)

    def full_green(self, SM):
        G, ov = mixed_density_matrix(self.PsiT, SM, compact=False)
        return G[:, None], ov

    def full_green_vbias(self, Gf, dt):
        """npol = 2: the diagonal polarization blocks, sum_p sum_ik L[i,k,n] G[w, pM+i, pM+k]."""
        W, M = Gf.shape[0], self.M
        g = Gf[:, 0, :M, :M] + Gf[:, 0, M:, M:]
        return math.sqrt(dt) * (g.reshape(W, M * M) @ self.Likn.reshape(M * M, self.Nc))

    def propagate(self, SM, P1, V, order):
        W, M2, N = SM.shape
        M = M2 // 2
        halves = np.ascontiguousarray(SM).reshape(2 * W, M, N)
        return propagate(halves, P1, np.repeat(V, 2, axis=0), order).reshape(W, M2, N)

    def vbias(self, G, dt):
        W = G.shape[0]
        return math.sqrt(dt) * (G.reshape(W, -1) @ self.Lnak.reshape(self.Nc, -1).T)

    def energy(self, G, addH1=True, addEJ=True, addEXX=True, chunk=None):
        W, N, M2 = G.shape
        Nc = self.Nc
        E = np.zeros((W, 3), dtype=np.complex128)
        if addH1:
            E[:, 0] = self.E0 + np.einsum('waj,aj->w', G, self.haj)
        if addEXX:
            T = (G.reshape(W * N, M2) @ self.Lnak.reshape(Nc * N, M2).T).reshape(W, N, Nc, N)  # T[w,b,n,a]
            E[:, 1] = -0.5 * np.einsum('wanb,wbna->w', T, T)
            if addEJ:
                Kl = np.einsum('wana->wn', T)
                E[:, 2] = 0.5 * np.einsum('wn,wn->w', Kl, Kl)
        return E


class MultiDetHamiltonian:
    """NOMSD with ndet > 1 determinants of one walker type (NOMSD.cpp:159-217,238-331,466-520).

    dets: one single-determinant Hamiltonian per determinant (Hamiltonian, CollinearHamiltonian or
    NoncollinearHamiltonian, each half-rotated with its own orbitals and built with ci = 1); ci: the
    coefficients.  The propagator (P1, vHS, propagation, orthogonalization) is that of the walker type.

      log overlap   a_d = log det_d + log(conj(ci_d)); log_m + log sum_d exp(a_d - log_m), log_m the
                    a_d of largest real part (Log_Overlap :301-331)
      force bias    the full G mixed over the determinants with weights conj(ci_d) exp(Ot_d - log_m),
                    log_m the walker's log overlap, then vbias on the full G with L itself (:238-278;
                    Real3IndexFactorization.hpp:392-426)
      energy        per determinant with its own haj / Lnak, mixed with conj(ci_d) exp(ov_d - log_m),
                    log_m the ov_d of largest real part (Energy :184-216)
      vMF           pairs p <= q of the trial's own determinants: G of PsiT_q against PsiT_p^H weighted
                    by Re(conj(ci_q) ci_p exp(log det)), normalised by the weights' sum (vMF :466-512)
      walkers       start as the determinant of largest |ci| (initial_guess :132-153)
    """

    def __init__(self, dets, ci):
        self.dets = list(dets)
        self.ci = np.asarray(ci, dtype=np.complex128)
        d0 = self.dets[0]
        self.M, self.Nc, self.E0, self.N = d0.M, d0.Nc, d0.E0, d0.N
        self.Likn, self.hcore = d0.Likn, d0.hcore

    def _lci(self, d):
        c = self.ci[d]
        return np.log(1e-12 if abs(c) < 1e-12 else np.conj(c))

    # the walker type's propagator
    def vHS(self, X, dt):
        return self.dets[0].vHS(X, dt)

    def one_body_propagator_matrix(self, dt, vMF):
        return self.dets[0].one_body_propagator_matrix(dt, vMF)

    def propagate(self, SM, P1, V, order):
        return self.dets[0].propagate(SM, P1, V, order)

    def orthogonalize(self, SM):
        return self.dets[0].orthogonalize(SM)

    def trial_walker(self):
        return self.dets[int(np.argmax(np.abs(self.ci)))].trial_walker()

    @staticmethod
    def _log_sum(a):
        """log sum_d exp(a[d, w]) per walker, about the a of largest real part."""
        out = np.empty(a.shape[1], np.complex128)
        for w in range(a.shape[1]):
            lm = a[int(np.argmax(a[:, w].real)), w]
            out[w] = lm + np.log(np.sum(np.exp(a[:, w] - lm)))
        return out

    def log_overlap(self, SM):
        a = np.stack([d.det_log_overlap(SM) + self._lci(i) for i, d in enumerate(self.dets)])
        return self._log_sum(a)

    def green(self, SM):
        log_m = self.log_overlap(SM)
        G = 0.0
        wsum = 0.0
        for i, d in enumerate(self.dets):
            Gd, ot = d.full_green(SM)
            wgt = np.conj(self.ci[i]) * np.exp(d.ov_factor * ot - log_m)
            wsum = wsum + wgt
            G = G + Gd * wgt[:, None, None, None]
        return G / wsum[:, None, None, None], log_m

    def vbias(self, G, dt):
        return self.dets[0].full_green_vbias(G, dt)

    def local_energy(self, SM):
        Es, ovs = [], []
        for d in self.dets:
            E, ov = d.local_energy(SM)
            Es.append(E)
            ovs.append(ov)
        Es, ovs = np.stack(Es), np.stack(ovs)
        W = SM.shape[0]
        E = np.empty((W, 3), np.complex128)
        Ov = np.empty(W, np.complex128)
        for w in range(W):
            lm = ovs[int(np.argmax(ovs[:, w].real)), w]
            e = np.exp(ovs[:, w] - lm) * np.conj(self.ci)
            deno = np.sum(e)
            E[w] = np.sum(e[:, None] * Es[:, w, :], axis=0) / deno
            Ov[w] = np.log(deno) + lm
        return E, Ov

    def mean_field(self, dt):
        Gsum = 0.0
        Osum = 0.0
        for p_, dp in enumerate(self.dets):
            B = dp.trial_walker()[None]
            for q_ in range(p_, len(self.dets)):
                Gq, ov = self.dets[q_].full_green(B)
                scl = (np.conj(self.ci[q_]) * self.ci[p_] * np.exp(ov[0])).real
                Osum += scl
                Gsum = Gsum + scl * Gq
        return self.vbias(Gsum / Osum, dt)[0].real.astype(np.complex128)


def trial_density(ham):
    """G of the trial against itself (NOMSD::vMF: MixedDensityMatrix(PsiT, PsiT^H), NOMSD.cpp:437-466)."""
    return ham.green(ham.trial_walker()[None])[0]


def vMF(ham, dt):
    """NOMSD::vMF (NOMSD.cpp:437-466) with zero_imag (AFQMCBasePropagator.cpp:107)."""
    return ham.mean_field(dt)


def hermitize(H):
    """math::hermitize (numerics/operations/tensor.hpp:75-93)."""
    H = np.array(H, dtype=np.complex128)
    n = H.shape[0]
    for i in range(n):
        H[i, i] = H[i, i].real
        for j in range(i + 1, n):
            H[i, j] = 0.5 * H[i, j] + 0.5 * np.conj(H[j, i])
            H[j, i] = np.conj(H[i, j])
    return H


def exp_hermitian(A):
    """math::exp_hermitian (exp.hpp:28-60): M sqrt(exp(V)) (M sqrt(exp(V)))^H."""
    V, Mv = np.linalg.eigh(np.asarray(A, dtype=np.complex128))
    Ms = Mv * np.sqrt(np.exp(V))[None, :]
    return Ms @ np.conj(Ms.T)


def build_P1(ham, vmf, dt, dense=False, drop=1e-8):
    """generateP1 (AFQMCBasePropagator.cpp:43-214): P1 = exp(-1/2 herm(H1)).

    With ``dense=False`` entries with |P1_ij| < drop are zeroed, which is what the CSR
    conversion ``to_csr(P1d, 1e-8)`` keeps (AFQMCBasePropagator.cpp:165-172).
    """
    H1 = ham.one_body_propagator_matrix(dt, vmf)
    H1 = hermitize(H1) * (-0.5)
    P = exp_hermitian(H1)
    if not dense:
        P = np.where(np.abs(P) < drop, 0.0, P)
    return P


def build_P1_inv(ham, vmf, dt, dense=False, drop=1e-8):
    """generateP1(Pinv = true) (AFQMCBasePropagator.cpp:148-172): exp(+1/2 herm(H1)), the inverse
    of P1 before the thresholding, thresholded like P1."""
    H1 = hermitize(ham.one_body_propagator_matrix(dt, vmf)) * 0.5
    P = exp_hermitian(H1)
    if not dense:
        P = np.where(np.abs(P) < drop, 0.0, P)
    return P


# --------------------------------------------------------------------------------------------
# Fields (construct_X_kernel.hpp:34-87; probit.h:58-136; AFQMCBasePropagator.cpp:324-336)
# --------------------------------------------------------------------------------------------
_PA = (-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
       1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00)
_PB = (-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
       6.680131188771972e+01, -1.328068155288572e+01)
_PC = (-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
       -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00)
_PD = (7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
       3.754408661907416e+00)


def probit(p):
    """Acklam's rational approximation of the inverse normal CDF (published coefficients)."""
    p = np.asarray(p, dtype=np.float64)
    out = np.zeros_like(p)
    lo = (p > 0) & (p < 0.02425)
    hi = (p > 0.97575) & (p < 1)
    mid = (p >= 0.02425) & (p <= 0.97575)
    with np.errstate(divide='ignore', invalid='ignore'):
        q = np.sqrt(-2 * np.log(np.where(lo, p, 0.5)))
        vlo = ((((((_PC[0] * q + _PC[1]) * q + _PC[2]) * q + _PC[3]) * q + _PC[4]) * q + _PC[5]) /
               ((((_PD[0] * q + _PD[1]) * q + _PD[2]) * q + _PD[3]) * q + 1))
        q = np.sqrt(-2 * np.log(1 - np.where(hi, p, 0.5)))
        vhi = -((((((_PC[0] * q + _PC[1]) * q + _PC[2]) * q + _PC[3]) * q + _PC[4]) * q + _PC[5]) /
                ((((_PD[0] * q + _PD[1]) * q + _PD[2]) * q + _PD[3]) * q + 1))
        q = p - 0.5
        r = q * q
        vmid = ((((((_PA[0] * r + _PA[1]) * r + _PA[2]) * r + _PA[3]) * r + _PA[4]) * r + _PA[5]) * q /
                (((((_PB[0] * r + _PB[1]) * r + _PB[2]) * r + _PB[3]) * r + _PB[4]) * r + 1))
    out = np.where(lo, vlo, out)
    out = np.where(hi, vhi, out)
    out = np.where(mid, vmid, out)
    out = np.where(p == 0, -np.inf, out)
    out = np.where(p == 1, np.inf, out)
    return out


def _clamp_c(z, bound):
    a = np.abs(z)
    with np.errstate(divide='ignore', invalid='ignore'):
        return np.where(a > bound, z / a * bound, z)


def assemble_X(vb, vmf, u, vbias_bound=50.0, free_projection=False):
    """construct_X_impl for continuous charge fields; returns (X, HW).

    HW is accumulated sequentially over m, as the host loop does
    (AFQMCBasePropagator.cpp:726-731).
    """
    vmf_t = _clamp_c(np.asarray(vmf, np.complex128), vbias_bound)[None, :]
    vb_t = _clamp_c(np.asarray(vb, np.complex128), vbias_bound)
    if free_projection:
        vdiff = np.zeros_like(vb_t)
    else:
        vdiff = 1j * (vb_t - vmf_t)
    X = probit(u) + vdiff
    terms = -vdiff * (X - 0.5 * vdiff)
    HW = np.zeros(X.shape[0], dtype=np.complex128)
    for m in range(X.shape[1]):
        HW += terms[:, m]
    return X, HW


def meanfield_factor(X, vmf):
    """AFQMCBasePropagator.cpp:335-336: -1/2 Re(vMF.vMF) + i X.vMF."""
    vmf = np.asarray(vmf, np.complex128)
    return -0.5 * np.dot(vmf, vmf).real + 1j * (X @ vmf)


# --------------------------------------------------------------------------------------------
# Propagation (propagate.hpp:45-70,247-298)
# --------------------------------------------------------------------------------------------
def apply_expM(V, S, order=6):
    S = S.copy()
    T1 = S.copy()
    for n in range(1, order + 1):
        T2 = (1j / n) * (V @ T1)
        S += T2
        T1 = T2
    return S


def propagate(Wk, P1, V, order=6):
    TMN = P1[None, :, :] @ Wk
    TMN = apply_expM(V, TMN, order)
    return P1[None, :, :] @ TMN


# --------------------------------------------------------------------------------------------
# Walker update and weight bound (WalkerSetUpdate.hpp:46-218)
# --------------------------------------------------------------------------------------------
class Walkers:
    """SoA view of WalkerSetBase for CLOSED walkers (WalkerSetBase.cpp:44-124)."""

    def __init__(self, SM, weight=None):
        self.SM = np.array(SM, dtype=np.complex128)        # (W, M, N)
        W = self.SM.shape[0]
        self.weight = np.ones(W, np.complex128) if weight is None else np.array(weight, np.complex128)
        self.phase = np.ones(W, np.complex128)
        self.pseudo_eloc = np.zeros(W, np.complex128)
        self.e1 = np.zeros(W, np.complex128)
        self.exx = np.zeros(W, np.complex128)
        self.ej = np.zeros(W, np.complex128)
        self.ovlp = np.zeros(W, np.complex128)
        self.theta = np.zeros(W, np.complex128)

    FIELDS = ('SM', 'weight', 'phase', 'pseudo_eloc', 'e1', 'exx', 'ej', 'ovlp', 'theta')

    def size(self):
        return self.SM.shape[0]

    def copy(self):
        c = Walkers(self.SM)
        for f in self.FIELDS:
            setattr(c, f, getattr(self, f).copy())
        return c

    # back propagation (WalkerSetBase::resize_bp, WalkerSetBase.cpp:331-385): the anchored walkers,
    # the field ring and the weight-factor history travel with each walker
    BP_FIELDS = ('SMN', 'fields', 'wfac')
    nbp = 0

    def copy_walker(self, src, dst):
        for f in self.FIELDS + (self.BP_FIELDS if self.nbp else ()):
            getattr(self, f)[dst] = getattr(self, f)[src]

    def enable_back_propagation(self, nbp, nchol):
        W = self.size()
        self.nbp, self.nhist, self.hist_pos = nbp, 3 * nbp, 0
        self.SMN = self.SM.copy()
        self.fields = np.zeros((W, nbp, nchol), np.complex128)
        self.wfac = np.ones((W, 3 * nbp), np.complex128)


def walker_update(wset, dt, Eshift, energy_offset, new_ovlp, mf, hw,
                  lower_cutoff_scale=1.0, upper_cutoff_scale=10.0,
                  hybrid=True, free_projection=False, use_cp_constraint=False,
                  new_energies=None):
    nw = wset.size()
    hi = Eshift + upper_cutoff_scale * math.sqrt(2.0 / dt)
    lo = Eshift - lower_cutoff_scale * math.sqrt(2.0 / dt)
    wfac = np.zeros(nw, np.complex128)  # the step's phase over the projection (WalkerSetUpdate.hpp:141-147)
    for i in range(nw):
        old_ovlp = complex(wset.ovlp[i])
        old_eloc = complex(wset.pseudo_eloc[i])
        scale = 1.0
        dtheta = 0.0
        if not free_projection:
            dtheta = new_ovlp[i].imag - old_ovlp.imag - mf[i].imag
            if use_cp_constraint:
                scale = 1.0 if math.cos(dtheta) > 0.0 else 0.0
            else:
                scale = max(0.0, math.cos(dtheta))
        wset.theta[i] = dtheta
        if hybrid:
            eloc = (mf[i] - hw[i] - (new_ovlp[i] - old_ovlp)) / dt + energy_offset
        else:
            eloc = new_energies[i, 0] + new_energies[i, 1] + new_energies[i, 2]
        eloc = complex(eloc)
        if not math.isfinite(eloc.real):
            wset.weight[i] = 0.0
            wset.phase[i] = 0.0
            eloc = old_eloc
        else:
            if not free_projection:
                eloc = complex(min(max(eloc.real, lo), hi), eloc.imag)
            eloc_eff = eloc if hybrid else 0.5 * (eloc + old_eloc)
            w = np.exp(-dt * (eloc_eff - Eshift))
            wfac[i] = (w / abs(w) / scale) if abs(scale) > np.finfo(np.float64).tiny else 0.0
            wset.weight[i] *= (scale * w) if free_projection else (scale * abs(w))
            wset.phase[i] *= w / abs(w)
        wset.pseudo_eloc[i] = eloc
        wset.ovlp[i] = new_ovlp[i]
    if wset.nbp:
        wset.wfac[:, wset.hist_pos] = wfac
    if not hybrid:
        wset.e1[:] = new_energies[:, 0]
        wset.exx[:] = new_energies[:, 1]
        wset.ej[:] = new_energies[:, 2]


def bound_walker_weights(wset, target_population, floor=100.0, fraction=0.1):
    max_w = max(floor, fraction * target_population)
    for i in range(wset.size()):
        a = abs(wset.weight[i])
        if a > max_w:
            wset.weight[i] *= max_w / a


# --------------------------------------------------------------------------------------------
# Orthogonalization (orthogonalize.hpp:135-169; determinants_impl.hpp:78-108)
# --------------------------------------------------------------------------------------------
def orthogonalize(Wk):
    """Householder QR of each walker (zgeqrf + zungqr on the transposed layout), then Q's
    columns scaled by sign(Re R_ii); returns (Q, log det R) with log det R accumulated the
    way log_determinant_from_geqrf does."""
    Wk = np.array(Wk, dtype=np.complex128)
    nw, M, N = Wk.shape
    ldet = np.zeros(nw, np.complex128)
    for w in range(nw):
        qr, tau, work, info = lapack.zgeqrf(Wk[w])
        scl = np.where(qr.diagonal()[:N].real < 0, -1.0, 1.0)
        for i in range(N):
            ldet[w] += np.log(complex(scl[i] * qr[i, i]) + SMALL)
        q, work, info = lapack.zungqr(qr[:, :N], tau)
        Wk[w] = q * scl[None, :]
    return Wk, ldet


# --------------------------------------------------------------------------------------------
# Population control (population_control.hpp:34-65,143-255), single rank
# --------------------------------------------------------------------------------------------
def comb(weights, r, num_target):
    weights = np.asarray(weights, dtype=np.float64)
    cum = np.empty_like(weights)
    acc = 0.0
    for i, w in enumerate(weights):       # std::partial_sum, sequential
        acc = acc + w
        cum[i] = acc
    total = cum[-1]
    if not total > 1e-6:
        raise RuntimeError(f"The total walker weight collapsed to {total}.")
    last = len(weights) - 1
    while weights[last] <= 0.0:
        last -= 1
    off = np.zeros(len(weights), dtype=np.int64)
    iw = 0
    ic = 0
    while ic < num_target:
        c = (ic + r) * total / num_target
        if c < cum[iw] or iw == last:
            off[iw] += 1
            ic += 1
        else:
            iw += 1
    return off


def copy_plan(offspring):
    """The (src, dst) walker copies swap_walkers_async performs on a single rank."""
    keep = list(int(k) for k in offspring)
    free = [i for i, k in enumerate(keep) if k == 0]
    plan = []
    nxt = 0
    for i, k in enumerate(keep):
        for _ in range(1, k):
            plan.append((i, free[nxt]))
            nxt += 1
    assert nxt == len(free)
    return plan


def plan_walker_exchange(offspring, counts):
    """plan_walker_exchange (population_control.hpp:73-133): (src rank, local walker, dst rank,
    copies) transfers for a rank-major population, rank r holding counts[r] walkers."""
    offspring = [int(k) for k in offspring]
    counts = [int(c) for c in counts]
    assert len(offspring) == sum(counts) and sum(offspring) == sum(counts)
    exports, deficits, first = [], [], 0
    for r, nw in enumerate(counts):
        local = offspring[first:first + nw]
        excess = sum(local) - nw
        if excess < 0:
            deficits.append([r, -excess])
        order = sorted(range(nw), key=lambda i: -local[i])  # std::stable_sort on copies, descending
        k = 0
        while excess > 0:
            m = min(local[order[k]], excess)
            exports.append([r, order[k], m])
            excess -= m
            k += 1
        first += nw
    plan, d = [], 0
    for src, walker, copies in exports:
        while copies > 0:
            n = min(copies, deficits[d][1])
            plan.append((src, walker, deficits[d][0], n))
            copies -= n
            deficits[d][1] -= n
            if deficits[d][1] == 0:
                d += 1
    return plan


def walker_moves(offspring, counts, rank):
    """rank's part of swap_walkers_async (population_control.hpp:143-209): sends (walker, dst) and
    receives (slot, src) in plan order, then the local copies (src slot, dst slot), the kept walkers'
    extra copies in index order before the received walkers'."""
    plan = plan_walker_exchange(offspring, counts)
    first = sum(counts[:rank])
    keep = [int(k) for k in offspring[first:first + counts[rank]]]
    for src, walker, dst, n in plan:
        if src == rank:
            keep[walker] -= n
    free = [i for i, k in enumerate(keep) if k == 0]
    nxt, sends, recvs, arrivals, copies = 0, [], [], [], []
    for src, walker, dst, n in plan:
        if src == rank:
            sends.append((walker, dst))
        elif dst == rank:
            recvs.append((free[nxt], src))
            arrivals.append((free[nxt], n))
            nxt += 1
    for slot, n in list(enumerate(keep)) + arrivals:
        for _ in range(1, n):
            copies.append((slot, free[nxt]))
            nxt += 1
    assert nxt == len(free)
    return sends, recvs, copies


def population_control(wset, r):
    weights = np.abs(wset.weight)
    off = comb(weights, r, wset.size())
    for src, dst in copy_plan(off):
        wset.copy_walker(src, dst)
    wset.weight = wset.weight / np.abs(wset.weight)
    return off


# --------------------------------------------------------------------------------------------
# Propagator + driver (AFQMCBasePropagator.cpp:290-392,736-741; run_afqmc.cpp:69-113)
# --------------------------------------------------------------------------------------------
class Propagator:
    def __init__(self, ham, dt, seed=0, taylor_order=6, vbias_bound=50.0,
                 lower_cutoff_scale=1.0, upper_cutoff_scale=10.0,
                 weight_bound_floor=100.0, weight_bound_fraction=0.1,
                 subtractMF=True, denseP1=False):
        self.ham = ham
        self.dt = dt
        self.seed = seed
        self.order = taylor_order
        self.vbias_bound = vbias_bound
        self.lower = lower_cutoff_scale
        self.upper = upper_cutoff_scale
        self.wfloor = weight_bound_floor
        self.wfrac = weight_bound_fraction
        self.vmf = vMF(ham, dt) if subtractMF else np.zeros(ham.Nc, np.complex128)
        self.denseP1 = denseP1
        self.P1 = build_P1(ham, self.vmf, dt, dense=denseP1)

    def propagate(self, wset, Eshift, step, target_population=None, uniforms=None):
        ham = self.ham
        W = wset.size()
        G, _ = ham.green(wset.SM)
        vb = ham.vbias(G, self.dt)
        if uniforms is None:
            uniforms = philox.uniforms(self.seed, philox.STREAM_FIELDS, step, W, ham.Nc)
        X, HW = assemble_X(vb, self.vmf, uniforms, self.vbias_bound)
        mf = meanfield_factor(X, self.vmf)
        if wset.nbp:
            wset.fields[:, wset.hist_pos % wset.nbp] = X  # storeFields (AFQMCBasePropagator.cpp:342-344)
        V = ham.vHS(X, self.dt)
        wset.SM = ham.propagate(wset.SM, self.P1, V, self.order)
        new_ov = ham.log_overlap(wset.SM)
        walker_update(wset, self.dt, Eshift, ham.E0, new_ov, mf, HW, self.lower, self.upper)
        tp = W if target_population is None else target_population
        bound_walker_weights(wset, tp, self.wfloor, self.wfrac)
        if wset.nbp:
            wset.hist_pos = (wset.hist_pos + 1) % wset.nhist
        return dict(G=G, vbias=vb, X=X, HW=HW, mf=mf, vHS=V, new_ovlp=new_ov)

    def orthogonalize(self, wset):
        wset.SM = self.ham.orthogonalize(wset.SM)
        wset.ovlp = self.ham.log_overlap(wset.SM)


def wfn_energy(ham, wset):
    """NOMSD::Energy(wset) (NOMSD.cpp:159-217 / :64-75): writes E1_, EXX_, EJ_, OVLP."""
    E, ov = ham.local_energy(wset.SM)
    wset.ovlp = ov
    wset.e1, wset.exx, wset.ej = E[:, 0].copy(), E[:, 1].copy(), E[:, 2].copy()
    return E, ov


def average_pseudo_energy(wset, dt):
    e = np.exp(dt * wset.pseudo_eloc)
    avg = np.sum(wset.weight * e) / np.sum(wset.weight)
    return math.log(avg.real) / dt


def average_energy(wset):
    return (np.sum(wset.weight * (wset.e1 + wset.exx + wset.ej)) / np.sum(wset.weight)).real


def measure_energy(ham, wset):
    """EnergyEstimator::measure: sum_w w E_w / sum_w w, plus the three components."""
    E, ov = wfn_energy_noupdate(ham, wset)
    wsum = np.sum(wset.weight)
    avg = (wset.weight @ E) / wsum
    return dict(Energy=complex(np.sum(avg)), OnebodyEnergy=complex(avg[0]),
                ExchangeEnergy=complex(avg[1]), CoulombEnergy=complex(avg[2]),
                TotalWeight=complex(wsum))


def wfn_energy_noupdate(ham, wset):
    return ham.local_energy(wset.SM)


def init_walkers(ham, wset):
    """execute.cpp:172-184: Energy(wset), seedPseudoEnergy, Eshift = averageEnergy."""
    wfn_energy(ham, wset)
    wset.pseudo_eloc = wset.e1 + wset.exx + wset.ej
    return average_energy(wset)


def run(ham, wset, prop, steps, Eshift, ortho_interval=10, pop_interval=10,
        equilibration_steps=100, measure_interval=10, relax=None, step0=0, record=None):
    """run_afqmc (run_afqmc.cpp:69-113). Returns (Eshift, list of measurements)."""
    if relax is None:
        relax = 1 - math.exp(-10.0 / equilibration_steps) if equilibration_steps > 1 else 1.0
    meas = []
    pop_calls = 0
    for step in range(step0, step0 + steps):
        prop.propagate(wset, Eshift, step)
        if step % ortho_interval == 0:
            prop.orthogonalize(wset)
        if step % pop_interval == 0:
            population_control(wset, philox.comb_uniform(prop.seed, step))
            pop_calls += 1
        if step >= equilibration_steps:
            if step % measure_interval == 0:
                meas.append((step, measure_energy(ham, wset)))
        else:
            Eshift += relax * (average_pseudo_energy(wset, prop.dt) - Eshift)
        if record is not None:
            record.append(dict(step=step, Eshift=Eshift, weight=wset.weight.copy(),
                               ovlp=wset.ovlp.copy(), pseudo_eloc=wset.pseudo_eloc.copy()))
    return Eshift, meas


# --------------------------------------------------------------------------------------------
# Seeded replay of one stage on the reference's own random streams (execute.cpp:117-190,
# run_afqmc.cpp:69-104, EnergyEstimator.h:51-100, Measurements.hpp:96-147), one rank
# --------------------------------------------------------------------------------------------
def measure_step(ham, wset, step, dt):
    """One bin of every observable EnergyEstimator::measure records at this step."""
    E, ov = wfn_energy_noupdate(ham, wset)
    w = wset.weight
    den = np.sum(w)                                 # MeasurementOutput's denominator
    avg = (w @ E) / den                             # gemv(transpose(E), weights)
    aw = np.abs(w)
    return {"Energy": complex(np.sum(avg)), "OnebodyEnergy": complex(avg[0]),
            "ExchangeEnergy": complex(avg[1]), "CoulombEnergy": complex(avg[2]),
            "Overlap": complex(np.sum(np.exp(ov) * w) / den),
            "ProjectionTime": (step + 1) * dt,
            "EffectiveNumWalkers": float(np.sum(aw) ** 2 / np.sum(aw * aw)),
            "Phase": complex(np.sum(w) / np.sum(aw)), "TotalWeight": complex(np.sum(w))}


def _references(ham):
    """(determinant Hamiltonians, coefficients) of a trial: NOMSD::getReferences (NOMSD.cpp:104-129)."""
    if isinstance(ham, MultiDetHamiltonian):
        return ham.dets, ham.ci
    return [ham], np.array([getattr(ham, "ci", 1.0)], np.complex128)


def _batched_full_green(A, B):
    """Per walker: T = A B (A (W, n, Mr) in the herm form), log det, and the full G = A^T T^-T B^T;
    an empty sector gives G = 0 and log det 0."""
    W, Mr, n = B.shape
    if n == 0:
        return np.zeros((W, Mr, Mr), np.complex128), np.zeros(W, np.complex128)
    T = A @ B
    ov = np.zeros(W, np.complex128)
    Tinv = np.empty_like(T)
    for w in range(W):
        ov[w], Tinv[w] = lu_logdet_inverse(T[w])
    Gc = np.transpose(Tinv, (0, 2, 1)) @ np.transpose(B, (0, 2, 1))
    return np.transpose(A, (0, 2, 1)) @ Gc, ov


def _walker_kind(det):
    if isinstance(det, NoncollinearHamiltonian):
        return "NONCOLLINEAR"
    return "COLLINEAR" if isinstance(det, CollinearHamiltonian) else "CLOSED"


def _rdm_reduce(parts, coeffs, w, wt, M):
    """OneRDM and the folded DiagonalTwoRDM (Observables/onerdm.hpp:42-75, diagonal_twordm.hpp:36-140)
    from per-reference full G's and walker coefficients, divided by sum_w w."""
    nspin, Mr = parts[0].shape[1], parts[0].shape[2]
    nblk = {"COLLINEAR": 3, "CLOSED": 2}.get(wt, 1)
    one = np.zeros((nspin, Mr, Mr), np.complex128)
    avg = np.zeros((nblk, Mr, Mr), np.complex128)
    for G, c in zip(parts, coeffs):
        wc = w * c
        one += np.einsum('w,wsij->sij', wc, G)
        dg = np.einsum('wsii->wsi', G)
        for sp in range(nspin):
            avg[2 * sp] += np.einsum('w,wi,wj->ij', wc, dg[:, sp], dg[:, sp])
            avg[2 * sp] -= np.einsum('w,wij,wji->ij', wc, G[:, sp], G[:, sp])
        if wt != "NONCOLLINEAR":
            avg[1] += np.einsum('w,wi,wj->ij', wc, dg[:, 0], dg[:, 1 if wt == "COLLINEAR" else 0])
    den = np.sum(w)
    one, avg = one / den, avg / den
    out = []
    if wt != "NONCOLLINEAR":
        for i in range(M):
            out += [(avg[0, i, j] + avg[0, j, i]) / 2 for j in range(i + 1, M)]
            out += [avg[1, i, j] for j in range(M)]
        if wt == "COLLINEAR":
            for i in range(M):
                out += [(avg[2, i, j] + avg[2, j, i]) / 2 for j in range(i + 1, M)]
    else:
        for i in range(2 * M):
            out += [(avg[0, i, j] + avg[0, j, i]) / 2 for j in range(i + 1, 2 * M)]
    return one, np.array(out, np.complex128)


def _observables_reduce(parts, coeffs, w, wt, M, two_rdm=True, spin_corr=True, pair_maps=None):
    """TwoRDM, SpinCorr and PairCorr (Observables/twordm.hpp:41-77, spincorr.hpp:36-136,
    paircorr.hpp:62-152) from per-reference full G's (W, nspin, R, R) and walker coefficients,
    divided by sum_w w.  TwoRDM: [block][i][k][j][l], blocks (a,a,a,a), (a,a,b,b), (b,b,b,b) (CLOSED:
    two); SpinCorr: (2, M(M+1)/2), the XY then the Z channel over i <= j; PairCorr: (npair, npair, M,
    M) for the maps (npair, M)."""
    out = {}
    den = np.sum(w)
    nspin = parts[0].shape[1]
    if two_rdm and wt != "NONCOLLINEAR":  # twordm.hpp:34-36
        avg = np.zeros((nspin + 1, M, M, M, M), np.complex128)
        for G, c in zip(parts, coeffs):
            XwG = (w * c)[:, None, None, None] * G
            for sp in range(nspin):
                avg[2 * sp] += np.einsum('wik,wjl->ikjl', XwG[:, sp], G[:, sp])
                avg[2 * sp] -= np.einsum('wil,wjk->ikjl', XwG[:, sp], G[:, sp])
            avg[1] += np.einsum('wik,wjl->ikjl', XwG[:, 0], G[:, nspin - 1])
        out["TwoRDM"] = avg / den
    if spin_corr:  # spincorr.hpp:58-124, term by term
        avg = np.zeros((2, M * (M + 1) // 2), np.complex128)
        for G, c in zip(parts, coeffs):
            Xw = w * c
            idx = 0
            for i in range(M):
                for j in range(i, M):
                    if wt in ("CLOSED", "COLLINEAR"):
                        Gu = G[:, 0]
                        Gd = G[:, 1] if wt == "COLLINEAR" else G[:, 0]
                        if j == i:
                            z = Gu[:, i, i] * (1.0 - Gd[:, j, j]) + Gd[:, i, i] * (1.0 - Gu[:, j, j])
                            xy = Gu[:, i, j] * (1.0 - Gd[:, j, i]) + Gd[:, i, j] * (1.0 - Gu[:, j, i])
                        else:
                            z = (Gu[:, i, i] * (Gu[:, j, j] - Gd[:, j, j]) + Gd[:, i, i] * (Gd[:, j, j] - Gu[:, j, j])
                                 - Gu[:, i, j] * Gu[:, j, i] - Gd[:, i, j] * Gd[:, j, i])
                            xy = Gu[:, i, j] * (-Gd[:, j, i]) + Gd[:, i, j] * (-Gu[:, j, i])
                    else:
                        g = G[:, 0]
                        I, J = i + M, j + M
                        if j == i:
                            z = (g[:, i, i] * (1.0 - g[:, J, J]) + g[:, I, I] * (1.0 - g[:, j, j])
                                 - g[:, i, J] * (-g[:, J, i]) - g[:, I, j] * (-g[:, j, I]))
                            xy = (g[:, i, j] * (1.0 - g[:, J, I]) + g[:, I, J] * (1.0 - g[:, j, i])
                                  + g[:, J, j] * g[:, i, I] + g[:, j, J] * g[:, I, i])
                        else:
                            z = (g[:, i, i] * (g[:, j, j] - g[:, J, J]) + g[:, I, I] * (g[:, J, J] - g[:, j, j])
                                 - g[:, i, j] * g[:, j, i] - g[:, I, J] * g[:, J, I]
                                 - g[:, i, J] * (-g[:, J, i]) - g[:, I, j] * (-g[:, j, I]))
                            xy = (g[:, i, j] * (-g[:, J, I]) + g[:, I, J] * -g[:, j, i]
                                  + g[:, J, j] * g[:, i, I] + g[:, j, J] * g[:, I, i])
                    avg[1, idx] += np.sum(Xw / 4.0 * z)
                    avg[0, idx] += np.sum(Xw / 2.0 * xy)
                    idx += 1
        out["SpinCorr"] = avg / den
    if pair_maps is not None and wt != "CLOSED":  # paircorr.hpp:37-40, 80-135
        maps = np.asarray(pair_maps, dtype=np.int64)
        n = maps.shape[0]
        avg = np.zeros((n, n, M, M), np.complex128)
        for G, c in zip(parts, coeffs):
            Xw = w * c
            for a in range(n):
                for b in range(n):
                    for i in range(M):
                        ib = maps[a, i]
                        if ib < 0:
                            continue
                        for j in (range(i + 1, M) if wt == "COLLINEAR" else range(M)):
                            jb = maps[b, j]
                            if jb < 0:
                                continue
                            if wt == "COLLINEAR":
                                Gup, Gdn = G[:, 0], G[:, 1]
                                cc = (Gup[:, i, j] * Gdn[:, ib, jb] + Gup[:, i, jb] * Gdn[:, ib, j]
                                      + Gdn[:, i, jb] * Gup[:, ib, j] + Gdn[:, i, j] * Gup[:, ib, jb])
                            else:
                                g = G[:, 0]
                                cc = (g[:, i, j] * g[:, M + ib, M + jb] - g[:, i, M + jb] * g[:, M + ib, j])
                                cc = cc + (g[:, i, jb] * g[:, M + ib, M + j] - g[:, i, M + j] * g[:, M + ib, jb])
                                cc = cc + (g[:, M + i, M + jb] * g[:, ib, j] - g[:, M + i, j] * g[:, ib, M + jb])
                                cc = cc + (g[:, M + i, M + j] * g[:, ib, jb] - g[:, M + i, jb] * g[:, ib, M + j])
                            avg[a, b, i, j] += np.sum(0.5 * Xw * cc)
        out["PairCorr"] = avg / den
    return out


class BackPropEstimator:
    """BackPropEstimator with the OneRDM and DiagonalTwoRDM observables (BackPropEstimator.hpp:36-275,
    AFQMCBasePropagator::BackPropagate :404-526), one rank.

    The walker set keeps, per walker, the anchored Slater matrices (SMN), a ring of the last nbp
    steps' fields and the history of the steps' weight factors (phase over projection).  When
    `bp` = step - anchor is one of the propagation lengths, every walker's copy of the trial's
    references is propagated backwards through the stored fields with the adjoint propagator
    (P1^H, exp(-i V^H), propagate.hpp:41-75 with TA = 'H'), orthogonalized every ortho_interval
    steps and at the end (the QR log dets summed in logdetR, shifted by their mean over references);
    the walker weights are restored by the last bp weight factors, and the RDMs are measured between
    the propagated references and the anchored walkers with coefficients conj(c_d) exp(ov_d +
    conj(logdetR_d)) / sum (CLOSED: both doubled).  The anchor moves to the current step once bp
    reaches the longest length."""

    def __init__(self, ham, prop, wset, steps=(2,), ortho_interval=10, path_restoration=True, observables=None):
        self.ham, self.prop = ham, prop
        self.observables = observables  # keyword arguments of _observables_reduce, or None
        self.steps = sorted(int(k) for k in steps)
        self.ortho = int(ortho_interval)
        self.path_restoration = path_restoration
        wset.enable_back_propagation(self.steps[-1], ham.Nc)
        self.anchor(wset, -1)

    def anchor(self, wset, step):
        wset.SMN = wset.SM.copy()
        self.bp_pos = step

    def measure(self, wset, step):
        bp = step - self.bp_pos
        out = self.back_propagate(wset, bp) if bp in self.steps else {}
        if bp >= self.steps[-1]:
            self.anchor(wset, step)
        return out

    def back_propagate(self, wset, nb):
        ham, prop = self.ham, self.prop
        dets, ci = _references(ham)
        W = wset.size()
        refs = [np.ascontiguousarray(np.broadcast_to(d.trial_walker(), (W,) + d.trial_walker().shape))
                for d in dets]
        logdetR = np.zeros((W, len(dets)), np.complex128)
        P1h = np.conj(prop.P1.T)
        slot = wset.hist_pos % wset.nbp
        for ni in range(nb - 1, -1, -1):
            slot = wset.nbp - 1 if slot == 0 else slot - 1
            V = ham.vHS(wset.fields[:, slot], prop.dt)
            Vadj = -np.conj(np.transpose(V, (0, 2, 1)))  # exp(i Vadj) = exp(-i V^H)
            for r in range(len(dets)):
                S = ham.propagate(refs[r], P1h, Vadj, prop.order)
                if ni == 0 or ni % self.ortho == 0:
                    S, ld = dets[0].orthogonalize_ldet(S)
                    logdetR[:, r] += ld
                refs[r] = S
        logdetR -= (logdetR.sum(axis=1) / len(dets))[:, None]
        weights = wset.weight.copy()
        if self.path_restoration:
            hpos = wset.hist_pos
            for _ in range(nb):
                hpos = wset.nhist - 1 if hpos == 0 else hpos - 1
                weights = weights * wset.wfac[:, hpos]
        f = dets[0].ov_factor
        parts, es = [], []
        for d, det in enumerate(dets):
            A = np.conj(np.transpose(refs[d], (0, 2, 1)))  # T = Refs^H SMN
            G, ov = det.bp_full_green(A, wset.SMN)
            parts.append(G)
            es.append(np.conj(ci[d]) * np.exp(f * ov + np.conj(f * logdetR[:, d])))
        tot = np.sum(es, axis=0)
        one, two = _rdm_reduce(parts, [e / tot for e in es], weights, _walker_kind(dets[0]), ham.M)
        pre = f"BackPropEstimator/Steps={nb}"
        out = {f"{pre}/OneRDM": one, f"{pre}/DiagonalTwoRDM": two}
        if self.observables:
            obs = _observables_reduce(parts, [e / tot for e in es], weights, _walker_kind(dets[0]), ham.M,
                                      **self.observables)
            out.update({f"{pre}/{k}": v for k, v in obs.items()})
        return out


def _spin_trials(ham):
    """Each spin block's trial (PsiT_s in the herm form) and its walker columns [c0, c1)."""
    if isinstance(ham, CollinearHamiltonian):
        return [(ham.PsiT_up, 0, ham.nup), (ham.PsiT_dn, ham.nup, ham.N)]
    return [(ham.PsiT, 0, ham.PsiT.shape[0])]


class TimeEvolvedBPEstimator:
    """TimeEvolvedBPEstimator with the mixed estimator's observables (TimeEvolvedBPEstimator.hpp:42-300,
    AFQMCBasePropagator::PropagateOperators :538-654), one rank, single- or multi-determinant trials.

    Per walker and spin, operator states X (-> c^+), Y (-> c) start from the identity and M from zero
    at the anchor.  At a measurement length bp the segment since the previous length is replayed from
    the stored fields, oldest first: X <- P1 e^{i vHS} P1 X and Y <- P1^-1 e^{i vHS^H} P1^-1 Y (the
    adjoint of the inverse propagator), then, with the walkers' current Slater matrices S:
    Y <- S S^H Y, M += Y^H X, X <- X - S S^H X.  The observables are measured on the dressed Green's
    functions G_s = M_s + (PsiT_s X_s)^T (Gc_s conj(Y_s)), Gc_s the walkers' compact mixed density
    matrix, per reference determinant d with its PsiT_d (constructTimeEvolvedMeasurementInputs,
    :48-140), with the walker weights restored over bp (2 bp with extra path restoration) steps and
    the coefficients conj(c_d) exp(f ov_d - OVLP) / sum_d' (...) (f = 2 for CLOSED, ov_d the sum
    over spins of the determinant's log overlaps with the current walkers): 1 for one determinant.
    The anchor moves to the current step once bp reaches the longest length."""

    def __init__(self, ham, prop, wset, steps=(2,), path_restoration=True, extra_path_restoration=False,
                 observables=None):
        self.ham, self.prop = ham, prop
        self.steps = sorted(int(k) for k in steps)
        self.restore = path_restoration or extra_path_restoration
        self.extra = extra_path_restoration
        self.observables = observables
        wset.enable_back_propagation(self.steps[-1], ham.Nc)
        self.P1inv = build_P1_inv(ham, prop.vmf, prop.dt, dense=prop.denseP1)
        self.anchor(wset, -1)

    def anchor(self, wset, step):
        W, R = wset.size(), wset.SM.shape[1]
        ns = len(_spin_trials(_references(self.ham)[0][0]))
        self.X = np.tile(np.eye(R, dtype=np.complex128), (ns, W, 1, 1))
        self.Y = self.X.copy()
        self.Mac = np.zeros_like(self.X)
        self.bp_pos = step

    def measure(self, wset, step):
        bp = step - self.bp_pos
        out = {}
        if bp in self.steps:
            i = self.steps.index(bp)
            self.evolve(wset, bp - (self.steps[i - 1] if i > 0 else 0))
            out = self._measure(wset, bp)
        if bp >= self.steps[-1]:
            self.anchor(wset, step)
        return out

    def evolve(self, wset, nsteps):
        ham, prop = self.ham, self.prop
        slot = (wset.hist_pos % wset.nbp + wset.nbp - nsteps) % wset.nbp
        for _ in range(nsteps):
            V = ham.vHS(wset.fields[:, slot], prop.dt)
            Vh = np.conj(np.transpose(V, (0, 2, 1)))
            for q in range(len(self.X)):
                self.X[q] = ham.propagate(self.X[q], prop.P1, V, prop.order)
                self.Y[q] = ham.propagate(self.Y[q], self.P1inv, Vh, prop.order)
            slot = (slot + 1) % wset.nbp
        for q, (_, c0, c1) in enumerate(_spin_trials(_references(ham)[0][0])):
            if c1 == c0:  # an empty sector: S S^H = 0
                self.Y[q] = 0.0
                continue
            S = wset.SM[:, :, c0:c1]
            Sh = np.conj(np.transpose(S, (0, 2, 1)))
            self.Y[q] = S @ (Sh @ self.Y[q])
            self.Mac[q] += np.conj(np.transpose(self.Y[q], (0, 2, 1))) @ self.X[q]
            self.X[q] = self.X[q] - S @ (Sh @ self.X[q])

    def _measure(self, wset, bp):
        ham = self.ham
        weights = wset.weight.copy()
        if self.restore:
            hpos = wset.hist_pos
            for _ in range(bp * (2 if self.extra else 1)):
                hpos = wset.nhist - 1 if hpos == 0 else hpos - 1
                weights = weights * wset.wfac[:, hpos]
        dets, ci = _references(ham)
        parts, es = [], []
        for d, det in enumerate(dets):
            blocks = []
            ov = np.zeros(wset.size(), np.complex128)
            for q, (P, c0, c1) in enumerate(_spin_trials(det)):
                G = self.Mac[q].copy()
                if c1 > c0:
                    Gc, ovq = mixed_density_matrix(P, wset.SM[:, :, c0:c1], compact=True)
                    G = G + np.transpose(P @ self.X[q], (0, 2, 1)) @ (Gc @ np.conj(self.Y[q]))
                    ov = ov + ovq
                blocks.append(G)
            parts.append(np.stack(blocks, axis=1))
            es.append(np.conj(ci[d]) * np.exp(det.ov_factor * ov - wset.ovlp))
        tot = np.sum(es, axis=0)
        coeffs = [e / tot for e in es]
        kind = _walker_kind(dets[0])
        one, two = _rdm_reduce(parts, coeffs, weights, kind, ham.M)
        pre = f"TimeEvolvedBP/Steps={bp}"
        out = {f"{pre}/OneRDM": one, f"{pre}/DiagonalTwoRDM": two}
        if self.observables:
            obs = _observables_reduce(parts, coeffs, weights, kind, ham.M, **self.observables)
            out.update({f"{pre}/{k}": v for k, v in obs.items()})
        return out


def measure_mixed_rdms(ham, wset, observables=None):
    """MixedEstimator::measure with the OneRDM and DiagonalTwoRDM observables (MixedEstimator.hpp:37-147),
    one rank: per reference determinant d the full mixed G_d and its log overlap (one determinant per
    spin, not doubled for CLOSED) give refCoeff_d = conj(c_d) exp(ov_d - OVLP) / sum_d' (...); the
    RDMs are the walker averages with weight * refCoeff_d (_rdm_reduce)."""
    dets, ci = _references(ham)
    parts = [d.full_green(wset.SM) for d in dets]
    e = [np.conj(ci[k]) * np.exp(ov - wset.ovlp) for k, (_, ov) in enumerate(parts)]
    tot = np.sum(e, axis=0)
    one, two = _rdm_reduce([G for G, _ in parts], [x / tot for x in e], wset.weight, _walker_kind(dets[0]), ham.M)
    out = {"MixedEstimator/OneRDM": one, "MixedEstimator/DiagonalTwoRDM": two}
    if observables:  # TwoRDM, SpinCorr, PairCorr (keyword arguments of _observables_reduce)
        obs = _observables_reduce([G for G, _ in parts], [x / tot for x in e], wset.weight, _walker_kind(dets[0]),
                                  ham.M, **observables)
        out.update({f"MixedEstimator/{k}": v for k, v in obs.items()})
    return out


def run_seeded(ham, nwalk, dt, steps, seed, ortho_interval=10, pop_interval=10, measure_interval=10,
               equilibration_steps=0, relax=None, rank=0, mixed_interval=None, bp_steps=None, bp_ortho_interval=None,
               observables=None, te_steps=None, te_extra_path_restoration=False, **prop_args):
    """execute_simulation + run_afqmc for one stage with HostRandomGenerator streams: walkers from
    the trial (NOMSD::initial_guess), Energy + seedPseudoEnergy, Eshift = averageEnergy, then the
    step loop.  Fields come from stream 1 (nwalk x nchol uniforms per step), the comb from stream 0.
    With mixed_interval the mixed estimator's one-body and diagonal two-body RDMs are measured too,
    with bp_steps (back propagation lengths) the back-propagated ones; observables (keyword
    arguments of _observables_reduce) adds TwoRDM, SpinCorr and PairCorr to both estimators; with
    te_steps the time-evolved back-propagation estimator runs (instead of bp_steps).
    Returns (initial Eshift, final Eshift, {observable: list of bins})."""
    from .mt19937 import HostRandomGenerator, split_seed
    walker_rng = HostRandomGenerator(split_seed(seed, rank, 0))
    field_rng = HostRandomGenerator(split_seed(seed, rank, 1))
    psi = ham.trial_walker()
    wset = Walkers(np.broadcast_to(psi, (nwalk,) + psi.shape))
    Eshift = init_walkers(ham, wset)
    E_init = Eshift
    prop = Propagator(ham, dt, **prop_args)
    bp = BackPropEstimator(ham, prop, wset, bp_steps, bp_ortho_interval or ortho_interval,
                           observables=observables) if bp_steps else None
    if te_steps:
        bp = TimeEvolvedBPEstimator(ham, prop, wset, te_steps, extra_path_restoration=te_extra_path_restoration,
                                    observables=observables)
    if relax is None:
        relax = 1 - math.exp(-10.0 / equilibration_steps) if equilibration_steps > 1 else 1.0
    series = {}
    for step in range(steps):
        u = field_rng.uniforms(nwalk * ham.Nc).reshape(nwalk, ham.Nc)
        prop.propagate(wset, Eshift, step, uniforms=u)
        if step % ortho_interval == 0:
            prop.orthogonalize(wset)
        if step % pop_interval == 0:
            population_control(wset, float(walker_rng.uniforms(1)[0]))
        if step >= equilibration_steps:
            if step % measure_interval == 0:
                for k, v in measure_step(ham, wset, step, dt).items():
                    series.setdefault(k, []).append(v)
            if mixed_interval and step % mixed_interval == 0:
                for k, v in measure_mixed_rdms(ham, wset, observables).items():
                    series.setdefault(k, []).append(v)
            if bp is not None:
                for k, v in bp.measure(wset, step).items():
                    series.setdefault(k, []).append(v)
        else:
            Eshift += relax * (average_pseudo_energy(wset, dt) - Eshift)
    return E_init, Eshift, series


def rebinned_average(series, rebinsize):
    """safiretools Results.average with a given rebin size (python/safiretools/results/stats.py:55-100,
    results.py:196-240): the series cut to whole bins, the mean of the bin means, and the standard
    error std(bins, ddof=1) / sqrt(bins) of real and imaginary parts separately."""
    s = np.asarray(series)
    nb = s.shape[0] // rebinsize
    if nb < 2:
        raise ValueError("fewer than two bins")
    bins = s[:nb * rebinsize].reshape(nb, rebinsize, *s.shape[1:]).mean(axis=1)
    mean = bins.mean(axis=0)
    if np.iscomplexobj(bins):
        err = (np.std(bins.real, axis=0, ddof=1) + 1j * np.std(bins.imag, axis=0, ddof=1)) / math.sqrt(nb)
    else:
        err = np.std(bins, axis=0, ddof=1) / math.sqrt(nb)
    return mean, err
