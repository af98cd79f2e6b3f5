// Serving loop: continuous batching of propagation blocks over device-resident systems.
//
// Each system owns an engine (its Hamiltonian tensors, trial and walkers resident in HBM, its own
// stream and block graphs).  Requests are blocks of run_afqmc steps for one system; the loop keeps
// at most max_inflight blocks on the GPU, one per system (a system's blocks are sequential: each
// continues from the previous one's walkers, step count and Eshift), and admits queued requests in
// arrival order as soon as a slot and the system are free, so requests that arrive while others
// run overlap with them on the device.  Engines are built on demand under the HBM budget; when it
// would be exceeded, idle engines are evicted least recently used first, their walkers and
// properties copied to the host and restored when the system is built again.
#include <chrono>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include "common.cuh"

namespace sfq {
namespace {
// electrons per walker: the rows of PsiT and the columns of a walker (COLLINEAR: up and down)
int electrons(const sfq_engine_params_t& p) {
  return p.nel + (p.walker_type == SFQ_WALKER_COLLINEAR ? p.nel_dn : 0);
}
// rows of a walker and columns of PsiT: nmo, or 2 nmo for NONCOLLINEAR spinors
int walker_rows(const sfq_engine_params_t& p) { return (p.walker_type == SFQ_WALKER_NONCOLLINEAR ? 2 : 1) * p.nmo; }

constexpr int kProps = 8;  // property columns of sfq_engine_get_walkers

struct SystemRec {
  sfq_engine_params_t p{};
  std::vector<double> hcore, Likn, PsiT;  // PsiT: complex (nel, nmo) as interleaved doubles
  sfq_engine_t eng = nullptr;
  size_t bytes = 0;          // device footprint of its engine (0 until first built)
  bool busy = false;         // a block is running
  bool started = false;      // walkers initialised (the trial energy and Eshift)
  unsigned long long next_step = 0;
  double Eshift = 0.0;
  double last_used = 0.0;
  std::vector<double> saved_SM, saved_props;  // walkers of an evicted engine
};

struct Request {
  int sys = 0;
  sfq_run_params_t rp{};
  int status = 1;  // 1 queued, 2 running, 0 done, else an error code
  double t_submit = 0, t_start = -1, t_finish = -1;
  unsigned long long step0 = 0;
  double Eshift = 0.0;
  std::vector<double> meas;
  int nmeas = 0;
  std::string message;
};

}  // namespace
}  // namespace sfq

struct sfq_server_s {
  sfq_server_params_t p{};
  std::vector<sfq::SystemRec> sys;
  std::vector<sfq::Request> req;
  std::deque<long long> queued;
  std::vector<long long> running;
  size_t used = 0;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace sfq {
namespace {

int evict(sfq_server_s& s, int keep, size_t need) {
  while (s.used + need > s.p.hbm_budget) {
    int victim = -1;
    for (int i = 0; i < (int)s.sys.size(); ++i) {
      const SystemRec& r = s.sys[i];
      if (i == keep || !r.eng || r.busy) continue;
      if (victim < 0 || r.last_used < s.sys[victim].last_used) victim = i;
    }
    if (victim < 0) return SFQ_ERR_OOM;  // everything resident is running: wait
    SystemRec& v = s.sys[victim];
    const size_t mn = size_t(walker_rows(v.p)) * electrons(v.p) * v.p.nwalk;
    v.saved_SM.resize(2 * mn);
    v.saved_props.resize(2 * size_t(kProps) * v.p.nwalk);
    int rc = sfq_engine_get_walkers(v.eng, v.saved_SM.data(), v.saved_props.data());
    if (rc) return rc;
    sfq_engine_destroy(v.eng);
    v.eng = nullptr;
    s.used -= v.bytes;
  }
  return SFQ_OK;
}

// build system i's engine (evicting others if the budget needs it) and bring its walkers back
int build(sfq_server_s& s, int i) {
  SystemRec& r = s.sys[i];
  if (r.eng) return SFQ_OK;
  int rc;
  if (r.bytes && (rc = evict(s, i, r.bytes))) return rc;
  sfq_engine_t e = nullptr;
  if ((rc = sfq_engine_create(&e, &r.p, r.hcore.data(), r.Likn.data(), r.PsiT.data()))) return rc;
  size_t b = 0;
  sfq_engine_footprint(e, &b);
  if (s.used + b > s.p.hbm_budget) {
    // first build of this system: now that its size is known, make room or give up for now
    if ((rc = evict(s, i, b))) {
      sfq_engine_destroy(e);
      r.bytes = b;
      return rc;
    }
  }
  r.eng = e;
  r.bytes = b;
  s.used += b;
  if (!r.started) {
    // execute.cpp:172-184: Energy, seedPseudoEnergy, Eshift = averageEnergy
    if ((rc = sfq_engine_energy(e, 1, nullptr))) return rc;
    if ((rc = sfq_engine_averages(e, nullptr, &r.Eshift, nullptr))) return rc;
    r.started = true;
  } else if (!r.saved_SM.empty()) {
    if ((rc = sfq_engine_set_walkers(e, r.saved_SM.data(), r.saved_props.data()))) return rc;
    r.saved_SM.clear();
    r.saved_props.clear();
  }
  return SFQ_OK;
}

}  // namespace
}  // namespace sfq

using namespace sfq;

extern "C" {

int sfq_server_create(sfq_server_t* out, const sfq_server_params_t* p) {
  if (!out || !p) return record_error(SFQ_ERR_ARG, "null pointer");
  if (p->max_inflight < 1 || p->hbm_budget == 0) return record_error(SFQ_ERR_ARG, "server: empty budget or slots");
  auto* s = new sfq_server_s();
  s->p = *p;
  *out = s;
  return SFQ_OK;
}

int sfq_server_destroy(sfq_server_t s) {
  if (!s) return SFQ_OK;
  for (auto& r : s->sys)
    if (r.eng) sfq_engine_destroy(r.eng);
  delete s;
  return SFQ_OK;
}

int sfq_server_add_system(sfq_server_t s, const sfq_engine_params_t* p, const double* hcore, const double* Likn,
                          const void* PsiT, int* id) {
  if (!s || !p || !hcore || !Likn || !PsiT || !id) return record_error(SFQ_ERR_ARG, "null pointer");
  if (p->nmo <= 0 || p->nel <= 0 || p->nchol <= 0 || p->nwalk <= 0)
    return record_error(SFQ_ERR_SHAPE, "server: invalid system sizes");
  SystemRec r;
  r.p = *p;
  r.p.device = s->p.device;
  const size_t MM = size_t(p->nmo) * p->nmo;
  r.hcore.assign(hcore, hcore + MM);
  r.Likn.assign(Likn, Likn + MM * p->nchol);
  const double* ps = static_cast<const double*>(PsiT);
  r.PsiT.assign(ps, ps + 2 * size_t(electrons(*p)) * walker_rows(*p));
  s->sys.push_back(std::move(r));
  *id = int(s->sys.size()) - 1;
  return SFQ_OK;
}

int sfq_server_warm(sfq_server_t s, int system) {
  if (!s || system < 0 || system >= (int)s->sys.size()) return record_error(SFQ_ERR_ARG, "server: no such system");
  const int rc = build(*s, system);
  if (rc == SFQ_ERR_OOM) return record_error(rc, "server: system %d does not fit in the HBM budget now", system);
  return rc;
}

int sfq_server_submit(sfq_server_t s, int system, const sfq_run_params_t* rp, long long* request) {
  if (!s || !rp || !request) return record_error(SFQ_ERR_ARG, "null pointer");
  if (system < 0 || system >= (int)s->sys.size()) return record_error(SFQ_ERR_ARG, "server: no such system");
  if (rp->steps <= 0) return record_error(SFQ_ERR_ARG, "server: a block needs steps");
  Request q;
  q.sys = system;
  q.rp = *rp;
  q.t_submit = s->now();
  s->req.push_back(q);
  *request = (long long)s->req.size() - 1;
  s->queued.push_back(*request);
  return SFQ_OK;
}

int sfq_server_progress(sfq_server_t s, int* completed) {
  if (!s) return record_error(SFQ_ERR_ARG, "null server");
  int done = 0;
  // retire finished blocks
  for (size_t k = 0; k < s->running.size();) {
    Request& q = s->req[s->running[k]];
    SystemRec& r = s->sys[q.sys];
    const int st = sfq_engine_block_query(r.eng);
    if (st == 0) {
      ++k;
      continue;
    }
    q.meas.assign(64 * 10, 0.0);
    int rc = st < 0 ? -st : sfq_engine_block_result(r.eng, &q.Eshift, q.meas.data(), 64, &q.nmeas);
    q.t_finish = s->now();
    q.status = rc;
    if (rc) q.message = sfq_last_error();
    q.meas.resize(size_t(10) * (q.nmeas < 64 ? q.nmeas : 64));
    if (!rc) {
      r.Eshift = q.Eshift;
      r.next_step += (unsigned long long)q.rp.steps;
    }
    r.busy = false;
    r.last_used = q.t_finish;
    s->running.erase(s->running.begin() + k);
    ++done;
  }
  // admit queued requests in arrival order, skipping those whose system is busy
  for (auto it = s->queued.begin(); it != s->queued.end() && (int)s->running.size() < s->p.max_inflight;) {
    Request& q = s->req[*it];
    SystemRec& r = s->sys[q.sys];
    if (r.busy) {
      ++it;
      continue;
    }
    int rc = build(*s, q.sys);
    if (rc == SFQ_ERR_OOM) break;  // no room until a running block finishes
    if (!rc) {
      sfq_run_params_t rp = q.rp;
      rp.step0 = r.next_step;
      q.step0 = r.next_step;
      rc = sfq_engine_block_async(r.eng, &rp, r.Eshift);
    }
    if (rc) {
      q.status = rc;
      q.message = sfq_last_error();
      q.t_finish = s->now();
      ++done;
    } else {
      q.status = 2;
      q.t_start = s->now();
      r.busy = true;
      r.last_used = q.t_start;
      s->running.push_back(*it);
    }
    it = s->queued.erase(it);
  }
  if (completed) *completed = done;
  return SFQ_OK;
}

int sfq_server_request(sfq_server_t s, long long request, sfq_request_info_t* info, double* meas, int max_meas) {
  if (!s || !info) return record_error(SFQ_ERR_ARG, "null pointer");
  if (request < 0 || request >= (long long)s->req.size()) return record_error(SFQ_ERR_ARG, "server: no such request");
  const Request& q = s->req[request];
  info->status = q.status;
  info->system = q.sys;
  info->t_submit = q.t_submit;
  info->t_start = q.t_start;
  info->t_finish = q.t_finish;
  info->Eshift = q.Eshift;
  info->nmeas = q.nmeas;
  info->step0 = q.step0;
  std::strncpy(info->message, q.message.c_str(), sizeof(info->message) - 1);
  info->message[sizeof(info->message) - 1] = 0;
  if (meas && q.status == 0) {
    const int n = q.nmeas < max_meas ? q.nmeas : max_meas;
    for (int k = 0; k < 10 * n; ++k) meas[k] = q.meas[k];
  }
  return SFQ_OK;
}

int sfq_server_stats(sfq_server_t s, size_t* used_bytes, int* resident, int* running, int* queued) {
  if (!s) return record_error(SFQ_ERR_ARG, "null server");
  if (used_bytes) *used_bytes = s->used;
  if (resident) {
    int n = 0;
    for (auto& r : s->sys) n += r.eng != nullptr;
    *resident = n;
  }
  if (running) *running = (int)s->running.size();
  if (queued) *queued = (int)s->queued.size();
  return SFQ_OK;
}

double sfq_server_clock(sfq_server_t s) { return s ? s->now() : 0.0; }

}  // extern "C"
