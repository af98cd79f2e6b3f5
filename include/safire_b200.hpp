// SAFIRE-B200 C++ interface: the reference's AFQMC class and function names, on top of the C ABI.
//
// Reference counterparts (SAFIRE source tree):
//   sfqmc::afqmc::det_ops::{MixedDensityMatrix, Log_Overlap, Propagate, orthogonalize}
//       src/AFQMC/SlaterDeterminantOperations/{density_matrix,propagate,orthogonalize}.hpp
//   sfqmc::afqmc::HamiltonianOperations / Real3IndexFactorization
//       src/AFQMC/HamiltonianOperations/HamiltonianOperations.h:34-103, Real3IndexFactorization.hpp
//   sfqmc::afqmc::WalkerSet (WalkerSetBase.h:51-572), AFQMCBasePropagator (AFQMCBasePropagator.h:51-172)
//
// Arrays are device pointers in the reference's C layouts; errors become safire_b200::Error,
// matching utils::check's throw-on-failure semantics (src/utilities/check.hpp:36-46).
#pragma once

#include <algorithm>
#include <complex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "safire_b200.h"

namespace safire_b200 {

using ComplexType = std::complex<double>;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != SFQ_OK) throw Error(rc, sfq_last_error());
}

// walker_data (WalkerConfig.hpp:28-48): the reference's names with the reference's values
enum walker_data {
  SM, UR, DR, VR, WEIGHT, PHASE, PSEUDO_ELOC_, E1_, EXX_, EJ_, OVLP, LOGSCL_UP, LOGSCL_DN, IS_UNITARY, SMN,
  FIELDS, WEIGHT_FAC, WEIGHT_HISTORY, THETA,
};
// the engine's property column of a walker_data id (sfq_engine_get_walkers order); the fields the
// engine does not keep as a property column are refused
inline int property_column(walker_data id) {
  switch (id) {
    case WEIGHT: return 0;
    case PHASE: return 1;
    case PSEUDO_ELOC_: return 2;
    case E1_: return 3;
    case EXX_: return 4;
    case EJ_: return 5;
    case OVLP: return 6;
    case THETA: return 7;
    default: throw Error(SFQ_ERR_ARG, "walker_data " + std::to_string(int(id)) + " is not a property column");
  }
}
// PropagatorTypes (propagator_types.hpp:13-20) and HamiltonianType (config.h:158-164)
enum PropagatorTypes {
  ContinuousChargePropagator, ContinuousSpinPropagator, DiscreteChargePropagator, DiscreteSpinPropagator,
  UndefinedPropagator,
};
enum class HamiltonianType { thc, kpthc, kp_factorized, real_dense_factorized, model_hamiltonian };

namespace det_ops {

// MixedDensityMatrix(A, B, C, ovlp, compact, herm = true)
inline void MixedDensityMatrix(const ComplexType* A, const ComplexType* B, ComplexType* C, ComplexType* ovlp,
                               int nwalk, int nmo, int nel, bool compact, void* ws, size_t ws_bytes,
                               void* stream = nullptr) {
  check(sfq_mixed_density_matrix(A, 1, B, C, ovlp, nwalk, nmo, nel, compact ? 1 : 0, ws, ws_bytes, stream));
}
inline void Log_Overlap(const ComplexType* A, const ComplexType* B, ComplexType* ovlp, int nwalk, int nmo, int nel,
                        void* ws, size_t ws_bytes, void* stream = nullptr) {
  check(sfq_log_overlap(A, 1, B, ovlp, nwalk, nmo, nel, ws, ws_bytes, stream));
}
// Propagate<DEVICE,'N'>(wset, P1, V, order) on the Slater matrices of CLOSED walkers
inline void Propagate(ComplexType* SM, const ComplexType* P1, const ComplexType* V, int nwalk, int nmo, int nel,
                      int order, void* ws, size_t ws_bytes, void* stream = nullptr) {
  check(sfq_propagate(SM, P1, 1, V, nwalk, nmo, nel, order, ws, ws_bytes, stream));
}
inline void orthogonalize(ComplexType* SM, ComplexType* log_detR, int nwalk, int nmo, int nel, void* ws,
                          size_t ws_bytes, void* stream = nullptr) {
  check(sfq_orthogonalize(SM, log_detR, nwalk, nmo, nel, ws, ws_bytes, stream));
}
inline size_t workspace_size(int op, int nwalk, int nmo, int nel, int nchol = 0) {
  return sfq_workspace_size(op, nwalk, nmo, nel, nchol);
}

}  // namespace det_ops

// population control planning on the host (population_control.hpp:34-209); no device needed
struct walker_transfer {
  int src;     // sending rank
  int walker;  // local index of the walker on src
  int dst;     // receiving rank
  int copies;  // copies of the walker that dst ends up with
};
// comb over |w| (host memory) with the uniform r: the copies of each walker
inline std::vector<int> comb(const std::vector<double>& weights, double r, int num_target) {
  std::vector<int> offspring(weights.size());
  check(sfq_comb_host(weights.data(), r, int(weights.size()), num_target, offspring.data()));
  return offspring;
}
inline std::vector<walker_transfer> plan_walker_exchange(const std::vector<int>& offspring,
                                                         const std::vector<int>& counts) {
  long ntot = 0;
  for (int c : counts) ntot += c;
  if (long(offspring.size()) != ntot)
    throw Error(SFQ_ERR_ARG, "plan_walker_exchange: offspring does not match the ranks' walkers");
  static_assert(sizeof(walker_transfer) == 4 * sizeof(int), "walker_transfer is the ABI's int quadruple");
  std::vector<walker_transfer> plan(size_t(ntot) + counts.size());
  int n = 0;
  check(sfq_plan_walker_exchange(offspring.data(), counts.data(), int(counts.size()),
                                 reinterpret_cast<int*>(plan.data()), int(plan.size()), &n));
  plan.resize(n);
  return plan;
}
// rank's part of swap_walkers_async: sends (walker, dst) and receives (slot, src) in plan order,
// then local copies (src slot, dst slot)
struct walker_moves_t {
  std::vector<std::pair<int, int>> sends, recvs, copies;
};
inline walker_moves_t walker_moves(const std::vector<int>& offspring, const std::vector<int>& counts, int rank) {
  long ntot = 0;
  for (int c : counts) ntot += c;
  if (long(offspring.size()) != ntot || rank < 0 || rank >= int(counts.size()))
    throw Error(SFQ_ERR_ARG, "walker_moves: offspring or rank does not match the ranks' walkers");
  static_assert(sizeof(std::pair<int, int>) == 2 * sizeof(int), "moves are the ABI's int pairs");
  int nw = counts[rank];
  walker_moves_t m;
  m.sends.resize(size_t(nw) + counts.size());
  m.recvs.resize(size_t(nw) + 1);
  m.copies.resize(size_t(nw) + 1);
  int ns = 0, nr = 0, nc = 0;
  check(sfq_walker_moves(offspring.data(), counts.data(), int(counts.size()), rank,
                         reinterpret_cast<int*>(m.sends.data()), int(m.sends.size()), &ns,
                         reinterpret_cast<int*>(m.recvs.data()), int(m.recvs.size()), &nr,
                         reinterpret_cast<int*>(m.copies.data()), int(m.copies.size()), &nc));
  m.sends.resize(ns);
  m.recvs.resize(nr);
  m.copies.resize(nc);
  return m;
}

// Real3IndexFactorization over caller-owned device tensors (CLOSED, ndet = 1)
class HamiltonianOperations {
 public:
  HamiltonianOperations(int nmo, int nel, int nchol, const double* Likn, const void* Lnak, bool lnak_complex,
                        const ComplexType* haj, double E0)
      : nmo_(nmo), nel_(nel), nchol_(nchol), Likn_(Likn), Lnak_(Lnak), lnak_complex_(lnak_complex), haj_(haj),
        E0_(E0) {}
  // with the one-body tensors too (device hcore and v0, nmo x nmo), for getOneBodyPropagatorMatrix
  HamiltonianOperations(int nmo, int nel, int nchol, const double* Likn, const void* Lnak, bool lnak_complex,
                        const ComplexType* haj, double E0, const double* hcore, const double* v0)
      : HamiltonianOperations(nmo, nel, nchol, Likn, Lnak, lnak_complex, haj, E0) {
    hcore_ = hcore;
    v0_ = v0;
  }

  int number_of_cholesky_vectors() const { return nchol_; }
  int number_of_ke_vectors() const { return nchol_; }
  double energy_offset() const { return E0_; }
  // (spin blocks, polarizations) of vHS: one of each for CLOSED walkers (Real3IndexFactorization.hpp:430-434)
  std::tuple<int, int> vHS_dims() const { return std::make_tuple(1, 1); }
  HamiltonianType getHamType() const { return HamiltonianType::real_dense_factorized; }
  // every Cholesky vector is a continuous charge field (Real3IndexFactorization.hpp:129-133)
  std::vector<int> getFieldTypes() const { return std::vector<int>(size_t(nchol_), int(ContinuousChargePropagator)); }
  // H1 = dt (h + v0) + vHS(vMF, dt) as a host [1][nmo][nmo] array (Real3IndexFactorization.hpp:99-124)
  std::vector<ComplexType> getOneBodyPropagatorMatrix(double dt, const std::vector<ComplexType>& vMF) const {
    if (!hcore_ || !v0_) throw Error(SFQ_ERR_ARG, "getOneBodyPropagatorMatrix: constructed without hcore and v0");
    if (long(vMF.size()) != nchol_) throw Error(SFQ_ERR_SHAPE, "getOneBodyPropagatorMatrix: Size mismatch");
    std::vector<double> v(vMF.size()), h(size_t(nmo_) * nmo_);
    for (size_t n = 0; n < vMF.size(); ++n) v[n] = vMF[n].real();
    check(sfq_one_body_matrix(hcore_, v0_, Likn_, v.data(), nmo_, nchol_, dt, h.data(), nullptr));
    return std::vector<ComplexType>(h.begin(), h.end());
  }

  // vbias(G, v, dt): v[W, nchol] = 2 sqrt(dt) G Lnak^T
  void vbias(const ComplexType* G, ComplexType* v, int nwalk, double dt, void* stream = nullptr) const {
    check(sfq_vbias(G, Lnak_, lnak_complex_ ? 1 : 0, v, nwalk, nel_, nmo_, nchol_, dt, 1, stream));
  }
  // vHS(X, dt): vHS[W, nmo, nmo] = sqrt(dt) sum_n L_n X_n
  void vHS(const ComplexType* X, ComplexType* vHS, int nwalk, double dt, void* stream = nullptr) const {
    check(sfq_vhs(Likn_, X, vHS, nwalk, nmo_, nchol_, dt, stream));
  }
  // energy(E, G, 0, addH1, addEJ, addEXX): E[W, 3] = (E1, EXX, EJ)
  void energy(ComplexType* E, const ComplexType* G, int nwalk, void* ws, size_t ws_bytes, bool addH1 = true,
              bool addEJ = true, bool addEXX = true, void* stream = nullptr) const {
    check(sfq_energy(E, G, haj_, Lnak_, lnak_complex_ ? 1 : 0, E0_, nwalk, nel_, nmo_, nchol_, addH1, addEJ, addEXX,
                     ws, ws_bytes, stream));
  }

 private:
  int nmo_, nel_, nchol_;
  const double* Likn_;
  const void* Lnak_;
  bool lnak_complex_;
  const ComplexType* haj_;
  double E0_;
  const double* hcore_ = nullptr;
  const double* v0_ = nullptr;
};

// The resident system: HamOps + NOMSD trial + WalkerSet + AFQMCBasePropagator on one GPU.
class Engine {
 public:
  Engine(const sfq_engine_params_t& p, const double* hcore, const double* Likn, const ComplexType* PsiT) {
    check(sfq_engine_create(&h_, &p, hcore, Likn, PsiT));
    p_ = p;
  }
  // a multi-determinant NOMSD trial: ndet matrices of the walker type's shape, coefficients ci
  Engine(const sfq_engine_params_t& p, const double* hcore, const double* Likn, int ndet, const ComplexType* PsiT,
         const ComplexType* ci) {
    check(sfq_engine_create_nomsd(&h_, &p, hcore, Likn, ndet, PsiT, ci));
    p_ = p;
  }
  ~Engine() { sfq_engine_destroy(h_); }
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;
  sfq_engine_t handle() const { return h_; }
  const sfq_engine_params_t& params() const { return p_; }
  // WalkerSet::resize: the engine rebuilt for n walkers, its walkers carried over round robin
  void resize(int n) {
    check(sfq_engine_resize(&h_, n));
    p_.nwalk = n;
  }

  // run_afqmc's loop as one device-resident block replayed from a CUDA graph (sfq_engine_block);
  // returns the measurements (10 doubles each), Eshift in/out
  std::vector<double> run_block(const sfq_run_params_t& rp, double& Eshift) {
    std::vector<double> meas(size_t(10) * 64);
    int n = 0;
    check(sfq_engine_block(h_, &rp, &Eshift, meas.data(), 64, &n));
    meas.resize(size_t(10) * (n < 64 ? n : 64));
    return meas;
  }
  // tile widths of the mixed-precision products: timed on this engine and kept, or set
  sfq_tiles_t autotune(int repeats = 9) {
    sfq_tiles_t t{};
    check(sfq_engine_autotune(h_, repeats, &t));
    return t;
  }
  void set_tiles(const sfq_tiles_t& t) { check(sfq_engine_set_tiles(h_, &t)); }

  // MixedEstimator's OneRDM (nspin, R, R) and folded DiagonalTwoRDM (see sfq_engine_measure_rdm)
  void measure_rdm(std::vector<ComplexType>& one_rdm, std::vector<ComplexType>& diag_two_rdm) {
    resize_rdms(one_rdm, diag_two_rdm);
    check(sfq_engine_measure_rdm(h_, one_rdm.data(), diag_two_rdm.data()));
  }
  // BackPropEstimator: the walker set's resize_bp, setAnchor and one back-propagated measurement
  void enable_back_propagation(int nbp) { check(sfq_engine_enable_back_propagation(h_, nbp)); }
  void bp_anchor() { check(sfq_engine_bp_anchor(h_)); }
  void measure_bp_rdm(int nsteps, int ortho_interval, bool path_restoration, std::vector<ComplexType>& one_rdm,
                      std::vector<ComplexType>& diag_two_rdm) {
    resize_rdms(one_rdm, diag_two_rdm);
    check(sfq_engine_measure_bp_rdm(h_, nsteps, ortho_interval, path_restoration ? 1 : 0, one_rdm.data(),
                                    diag_two_rdm.data()));
  }

 private:
  void resize_rdms(std::vector<ComplexType>& one, std::vector<ComplexType>& two) const {
    const long M = p_.nmo;
    const bool coll = p_.walker_type == SFQ_WALKER_COLLINEAR, ncol = p_.walker_type == SFQ_WALKER_NONCOLLINEAR;
    const long R = (ncol ? 2 : 1) * M;
    one.resize(size_t((coll ? 2 : 1) * R * R));
    two.resize(size_t(M * (2 * M - 1) - ((coll || ncol) ? 0 : M * (M - 1) / 2)));
  }
  sfq_engine_t h_ = nullptr;
  sfq_engine_params_t p_{};
};

// Several engines advanced together: one block of every member per CUDA graph launch
class EngineGroup {
 public:
  explicit EngineGroup(const std::vector<Engine*>& members) {
    std::vector<sfq_engine_t> hs;
    for (Engine* e : members) hs.push_back(e->handle());
    check(sfq_group_create(&g_, hs.data(), int(hs.size())));
    n_ = int(hs.size());
  }
  ~EngineGroup() { sfq_group_destroy(g_); }
  EngineGroup(const EngineGroup&) = delete;
  EngineGroup& operator=(const EngineGroup&) = delete;
  void set_lanes(int lanes) { check(sfq_group_set_lanes(g_, lanes)); }
  // rps and Eshift per member (Eshift in/out); status per member; measurements at 10 * 64 * i
  std::vector<double> run_block(const std::vector<sfq_run_params_t>& rps, std::vector<double>& Eshift,
                                std::vector<int>& status, std::vector<int>& nmeas) {
    std::vector<double> meas(size_t(10) * 64 * n_);
    status.assign(n_, 0);
    nmeas.assign(n_, 0);
    check(sfq_group_block(g_, rps.data(), Eshift.data(), status.data(), meas.data(), 64, nmeas.data()));
    return meas;
  }

 private:
  sfq_group_t g_ = nullptr;
  int n_ = 0;
};

// The request loop over resident systems (sfq_server_*)
class Server {
 public:
  explicit Server(const sfq_server_params_t& p) { check(sfq_server_create(&s_, &p)); }
  ~Server() { sfq_server_destroy(s_); }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  int add_system(const sfq_engine_params_t& p, const double* hcore, const double* Likn, const ComplexType* PsiT) {
    int id = -1;
    check(sfq_server_add_system(s_, &p, hcore, Likn, PsiT, &id));
    return id;
  }
  long long submit(int system, const sfq_run_params_t& rp) {
    long long rid = -1;
    check(sfq_server_submit(s_, system, &rp, &rid));
    return rid;
  }
  int progress() {
    int n = 0;
    check(sfq_server_progress(s_, &n));
    return n;
  }
  sfq_request_info_t request(long long rid, std::vector<double>* meas = nullptr) {
    sfq_request_info_t info{};
    std::vector<double> m(size_t(10) * 64);
    check(sfq_server_request(s_, rid, &info, m.data(), 64));
    if (meas) *meas = m;
    return info;
  }

 private:
  sfq_server_t s_ = nullptr;
};

// the auxiliary-field generator of an engine: counter-based Philox draws keyed by (seed, step,
// walker, vector), the stream sampleUniformFields stands for (Random.hpp:37-118)
class RandomGenerator {
 public:
  RandomGenerator(unsigned long long seed, int nwalk, int nchol) : seed_(seed), nwalk_(nwalk), nchol_(nchol) {}
  unsigned long long seed() const { return seed_; }
  // the uniforms of one step into a device buffer of nwalk x nchol doubles
  void sampleUniformFields(double* dev, unsigned long long step, void* stream = nullptr) const {
    check(sfq_field_uniforms(dev, seed_, step, nwalk_, nchol_, stream));
  }

 private:
  unsigned long long seed_;
  int nwalk_, nchol_;
};

// WalkerSet view of an engine (WalkerSetBase.h:51-572): size, properties, Slater matrices, copies
class WalkerSet {
 public:
  explicit WalkerSet(Engine& e) : e_(e) {}
  int size() const { return e_.params().nwalk; }
  std::vector<ComplexType> getProperty(walker_data id) const {
    const int col = property_column(id);
    std::vector<ComplexType> props(size_t(8) * size());
    check(sfq_engine_get_walkers(e_.handle(), nullptr, props.data()));
    return std::vector<ComplexType>(props.begin() + size_t(col) * size(), props.begin() + size_t(col + 1) * size());
  }
  // setProperty (WalkerSetBase.h:476-481): v holds at least size() values
  void setProperty(walker_data id, const std::vector<ComplexType>& v) {
    const int col = property_column(id);
    if (long(v.size()) < size()) throw Error(SFQ_ERR_SHAPE, "setProperty: Shape mismatch");
    std::vector<ComplexType> props(size_t(8) * size());
    check(sfq_engine_get_walkers(e_.handle(), nullptr, props.data()));
    std::copy(v.begin(), v.begin() + size(), props.begin() + size_t(col) * size());
    check(sfq_engine_set_walkers(e_.handle(), nullptr, props.data()));
  }
  std::vector<ComplexType> SlaterMatrices() const {
    const auto& p = e_.params();
    std::vector<ComplexType> sm(size_t(p.nwalk) * p.nmo * p.nel);
    check(sfq_engine_get_walkers(e_.handle(), sm.data(), nullptr));
    return sm;
  }
  void copy_walker(int from, int to) { check(sfq_engine_copy_walker(e_.handle(), from, to)); }
  void resize(int n) { e_.resize(n); }
  RandomGenerator getRNG() const {
    const auto& p = e_.params();
    return RandomGenerator(p.seed, p.nwalk, p.nchol);
  }
  Engine& engine() { return e_; }

 private:
  Engine& e_;
};

// AFQMCBasePropagator (AFQMCBasePropagator.h:51-172): Propagate / Orthogonalize on the engine
class AFQMCBasePropagator {
 public:
  explicit AFQMCBasePropagator(Engine& e) : e_(e) {}
  // nt is the time slice of finite-temperature walkers (WalkerSet::setTauStep); zero-temperature
  // walkers ignore it.  The fields of each call are those of the next step of the generator.
  void Propagate(WalkerSet& wset, double Eshift, int nt = 0) {
    (void)nt;
    check(sfq_engine_propagate(wset.engine().handle(), Eshift, step_++, nullptr));
  }
  void Orthogonalize(WalkerSet& wset) { check(sfq_engine_orthogonalize(wset.engine().handle())); }
  bool stores_local_energy() const { return false; }  // hybrid propagation
  // uniforms drawn per walker (at least nchol, AFQMCBasePropagator.cpp:708): the counter-based fields
  // are keyed per (walker, vector), so the block size changes no field
  void set_rng_block_size(int sz) {
    if (sz < e_.params().nchol) throw Error(SFQ_ERR_ARG, "set_rng_block_size: rng_block_size < nCV");
    rng_block_size_ = sz;
  }
  int rng_block_size() const { return rng_block_size_; }

 private:
  Engine& e_;
  unsigned long long step_ = 0;
  int rng_block_size_ = 0;
};

}  // namespace safire_b200
