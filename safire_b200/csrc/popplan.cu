// Host-side planning of population control over walkers sharded across ranks.  No CUDA call is
// made here: these entry points run on the host of every rank and need no device.
//
//   sfq_comb_host           comb over the gathered |w| (population_control.hpp:34-65), on the root
//   sfq_plan_walker_exchange the transfers between ranks (population_control.hpp:73-133)
//   sfq_walker_moves        one rank's sends, receives and local copies (population_control.hpp:143-209)
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"

using sfq::record_error;

namespace {

struct Transfer {
  int src, walker, dst, copies;
};

int check_population(const int* offspring, const int* counts, int nranks, long* ntot_out) {
  if (nranks <= 0) return record_error(SFQ_ERR_SHAPE, "plan_walker_exchange: %d ranks", nranks);
  if (!offspring || !counts) return record_error(SFQ_ERR_ARG, "plan_walker_exchange: null pointer");
  long ntot = 0;
  for (int r = 0; r < nranks; ++r) {
    if (counts[r] < 0) return record_error(SFQ_ERR_SHAPE, "plan_walker_exchange: rank %d holds %d walkers", r, counts[r]);
    ntot += counts[r];
  }
  long copies = 0;
  for (long i = 0; i < ntot; ++i) {
    if (offspring[i] < 0) return record_error(SFQ_ERR_ARG, "plan_walker_exchange: walker %ld has %d copies", i, offspring[i]);
    copies += offspring[i];
  }
  if (copies != ntot)
    return record_error(SFQ_ERR_ARG, "plan_walker_exchange: offspring does not preserve the population (%ld copies of %ld)",
                        copies, ntot);
  *ntot_out = ntot;
  return SFQ_OK;
}

// The plan: ranks with excess export their walkers with the most copies first (ties in index
// order), the exports filling the ranks with a deficit in rank order; an export splits only where
// a deficit runs out.  Deterministic, so every rank computes the same plan.
std::vector<Transfer> plan(const int* offspring, const int* counts, int nranks) {
  std::vector<Transfer> exports;
  std::vector<std::pair<int, int>> deficit;  // (rank, missing copies)
  std::vector<int> idx;
  long first = 0;
  for (int r = 0; r < nranks; first += counts[r], ++r) {
    const int* mine = offspring + first;
    int nw = counts[r];
    long held = 0;
    for (int i = 0; i < nw; ++i) held += mine[i];
    long excess = held - nw;
    if (excess < 0) deficit.push_back({r, int(-excess)});
    if (excess <= 0) continue;
    idx.resize(nw);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return mine[a] > mine[b]; });
    for (int k = 0; excess > 0; ++k) {
      int m = int(std::min<long>(mine[idx[k]], excess));
      exports.push_back({r, idx[k], -1, m});
      excess -= m;
    }
  }
  std::vector<Transfer> out;
  size_t d = 0;
  for (Transfer e : exports) {
    while (e.copies > 0) {
      int n = std::min(e.copies, deficit[d].second);
      out.push_back({e.src, e.walker, deficit[d].first, n});
      e.copies -= n;
      if ((deficit[d].second -= n) == 0) ++d;
    }
  }
  return out;
}

}  // namespace

extern "C" {

int sfq_comb_host(const double* weights, double r, int nwalk, int num_target, int* offspring) {
  if (nwalk <= 0 || num_target < 0) return record_error(SFQ_ERR_SHAPE, "comb: %d walkers, target %d", nwalk, num_target);
  if (!weights || !offspring) return record_error(SFQ_ERR_ARG, "comb: null pointer");
  if (!(r >= 0.0 && r < 1.0)) return record_error(SFQ_ERR_ARG, "comb uniform %g outside [0, 1)", r);
  // the running sum in walker order, as std::partial_sum forms it
  std::vector<double> cum(nwalk);
  double s = 0.0;
  for (int i = 0; i < nwalk; ++i) {
    if (!(weights[i] >= 0.0)) return record_error(SFQ_ERR_NONFINITE, "comb: |w| of walker %d is %g", i, weights[i]);
    cum[i] = (s += weights[i]);
  }
  double total = cum[nwalk - 1];
  if (!(total > 1e-6)) return record_error(SFQ_ERR_WEIGHT_COLLAPSE, "The total walker weight collapsed to %g.", total);
  int last = nwalk - 1;
  while (weights[last] <= 0.0) --last;  // total > 0, so some walker has weight
  std::fill(offspring, offspring + nwalk, 0);
  int iw = 0;
  for (int ic = 0; ic < num_target;) {
    if ((ic + r) * total / num_target < cum[iw] || iw == last) {
      ++offspring[iw];
      ++ic;
    } else {
      ++iw;
    }
  }
  return SFQ_OK;
}

int sfq_plan_walker_exchange(const int* offspring, const int* counts, int nranks, int* transfers, int capacity,
                             int* ntransfers) {
  long ntot = 0;
  if (int rc = check_population(offspring, counts, nranks, &ntot)) return rc;
  if (!ntransfers || (capacity > 0 && !transfers)) return record_error(SFQ_ERR_ARG, "plan_walker_exchange: null pointer");
  std::vector<Transfer> p = plan(offspring, counts, nranks);
  *ntransfers = int(p.size());
  if (int(p.size()) > capacity)
    return record_error(SFQ_ERR_WORKSPACE, "plan_walker_exchange: %zu transfers, room for %d", p.size(), capacity);
  for (size_t k = 0; k < p.size(); ++k) {
    transfers[4 * k + 0] = p[k].src;
    transfers[4 * k + 1] = p[k].walker;
    transfers[4 * k + 2] = p[k].dst;
    transfers[4 * k + 3] = p[k].copies;
  }
  return SFQ_OK;
}

int sfq_walker_moves(const int* offspring, const int* counts, int nranks, int rank, int* sends, int max_sends,
                     int* nsends, int* recvs, int max_recvs, int* nrecvs, int* copies, int max_copies, int* ncopies) {
  long ntot = 0;
  if (int rc = check_population(offspring, counts, nranks, &ntot)) return rc;
  if (rank < 0 || rank >= nranks) return record_error(SFQ_ERR_ARG, "walker_moves: rank %d of %d", rank, nranks);
  if (!nsends || !nrecvs || !ncopies) return record_error(SFQ_ERR_ARG, "walker_moves: null pointer");
  if ((max_sends > 0 && !sends) || (max_recvs > 0 && !recvs) || (max_copies > 0 && !copies))
    return record_error(SFQ_ERR_ARG, "walker_moves: null pointer");
  int nw = counts[rank];
  long first = 0;
  for (int r = 0; r < rank; ++r) first += counts[r];
  std::vector<Transfer> p = plan(offspring, counts, nranks);
  // copies each local walker keeps here once its exports are sent
  std::vector<int> keep(offspring + first, offspring + first + nw);
  for (const Transfer& t : p)
    if (t.src == rank) keep[t.walker] -= t.copies;
  std::vector<int> freed;  // slots of walkers with no copy left here, in index order
  for (int i = 0; i < nw; ++i)
    if (keep[i] == 0) freed.push_back(i);
  size_t next = 0;
  int ns = 0, nr = 0, nc = 0;
  *nsends = *nrecvs = *ncopies = 0;
  // the lists' lengths are counted first, so an undersized array is reported before anything is written
  {
    int need_s = 0, need_r = 0;
    for (const Transfer& t : p) {
      if (t.src == rank) ++need_s;
      else if (t.dst == rank) ++need_r;
    }
    const int need_c = int(freed.size()) - need_r;  // every freed slot not taken by a receive is a copy
    if (need_s > max_sends || need_r > max_recvs || need_c > max_copies) {
      *nsends = need_s;
      *nrecvs = need_r;
      *ncopies = need_c < 0 ? 0 : need_c;
      return record_error(SFQ_ERR_WORKSPACE, "walker_moves: %d sends, %d receives, %d copies; room for %d, %d, %d",
                          need_s, need_r, need_c, max_sends, max_recvs, max_copies);
    }
  }
  std::vector<std::pair<int, int>> arrivals;  // (slot, copies) of the walkers received
  // the sends and receives in plan order: both ends post them in the same order
  for (const Transfer& t : p) {
    if (t.src == rank) {
      sends[2 * ns + 0] = t.walker;
      sends[2 * ns + 1] = t.dst;
      ++ns;
    } else if (t.dst == rank) {
      if (next >= freed.size()) return record_error(SFQ_ERR_INTERNAL, "walker_moves: no free slot for a received walker");
      int slot = freed[next++];
      recvs[2 * nr + 0] = slot;
      recvs[2 * nr + 1] = t.src;
      ++nr;
      arrivals.push_back({slot, t.copies});
    }
  }
  // then the local copies: the kept walkers' extra copies in index order, then the received ones'
  auto replicate = [&](int src, int n) -> bool {
    for (int c = 1; c < n; ++c) {
      if (next >= freed.size()) return false;
      copies[2 * nc + 0] = src;
      copies[2 * nc + 1] = freed[next++];
      ++nc;
    }
    return true;
  };
  for (int i = 0; i < nw; ++i)
    if (!replicate(i, keep[i])) return record_error(SFQ_ERR_INTERNAL, "walker_moves: more copies than free slots");
  for (auto& a : arrivals)
    if (!replicate(a.first, a.second)) return record_error(SFQ_ERR_INTERNAL, "walker_moves: more copies than free slots");
  if (next != freed.size())
    return record_error(SFQ_ERR_INTERNAL, "walker_moves: %zu slots left unfilled", freed.size() - next);
  *nsends = ns;
  *nrecvs = nr;
  *ncopies = nc;
  return SFQ_OK;
}

}  // extern "C"
