// Elementwise / per-walker kernels of the propagation step: field assembly, walker update and
// weight bound, comb population control, energy reductions, and small layout helpers.
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "philox.cuh"
#include "probit.cuh"

namespace sfq {

namespace {

constexpr int RT = 256;

template <int NT>
__device__ __forceinline__ cplx block_sum(cplx v, cplx* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, off);
    v.y += __shfl_down_sync(0xffffffffu, v.y, off);
  }
  if (lane == 0) red[warp] = v;
  __syncthreads();
  cplx r = mk(0.0, 0.0);
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; ++i) r = cadd(r, red[i]);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

__device__ __forceinline__ cplx clamp_c(cplx z, double bound) {
  double a = hypot(z.x, z.y);
  if (a > bound) return mk(z.x / a * bound, z.y / a * bound);
  return z;
}

// construct_X_impl for continuous charge fields (construct_X_kernel.hpp:34-87) plus the
// meanfield factor (AFQMCBasePropagator.cpp:335-336); one CTA per walker, deterministic sums.
__global__ void __launch_bounds__(RT) assemble_x_kernel(cplx* X, const double* vmf, cplx* hw, cplx* mf,
                                                        FieldParams p) {
  __shared__ cplx red[RT / 32];
  const int w = blockIdx.x;
  const int Nc = p.nchol;
  cplx* Xw = X + (long)w * Nc;
  cplx acc_hw = mk(0.0, 0.0), acc_xv = mk(0.0, 0.0);
  double acc_v2 = 0.0;
  const int npair = (Nc + 1) / 2;
  for (int j = threadIdx.x; j < npair; j += RT) {
    double u[2];
    if (p.uniforms) {
      u[0] = p.uniforms[(long)w * Nc + 2 * j];
      u[1] = (2 * j + 1 < Nc) ? p.uniforms[(long)w * Nc + 2 * j + 1] : 0.5;
    } else {
      field_uniform_pair(p.seed, p.step_dev ? *p.step_dev : p.step, (uint32_t)w, (uint32_t)j, u[0], u[1]);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = 2 * j + h;
      if (n >= Nc) break;
      const double v0 = vmf[n];
      const double vmf_t = fabs(v0) > p.vbias_bound ? (v0 / fabs(v0)) * p.vbias_bound : v0;
      const cplx vb_t = clamp_c(Xw[n], p.vbias_bound);
      cplx vdiff = p.free_projection ? mk(0.0, 0.0) : mk(-(vb_t.y), vb_t.x - vmf_t);  // i*(vb - vmf)
      cplx x = mk(probit(u[h]) + vdiff.x, vdiff.y);
      Xw[n] = x;
      // -vdiff * (x - 0.5 vdiff)
      cplx t = cmul(vdiff, mk(x.x - 0.5 * vdiff.x, x.y - 0.5 * vdiff.y));
      acc_hw = csub(acc_hw, t);
      acc_xv = cadd(acc_xv, cscale(x, v0));
      acc_v2 += v0 * v0;
    }
  }
  cplx shw = block_sum<RT>(acc_hw, red);
  cplx sxv = block_sum<RT>(acc_xv, red);
  cplx sv2 = block_sum<RT>(mk(acc_v2, 0.0), red);
  if (threadIdx.x == 0) {
    hw[w] = shw;
    // -1/2 Re(vMF.vMF) + i * (X.vMF)
    mf[w] = mk(-0.5 * sv2.x - sxv.y, sxv.x);
  }
}

// walker_update + bound_local_energy + bound_walker_weights (WalkerSetUpdate.hpp:46-218)
__global__ void walker_update_kernel(WalkerProps wp, const cplx* new_ovlp, const cplx* mf, const cplx* hw,
                                     const cplx* E3, UpdateParams p, unsigned long long* stats) {
  const double Eshift = p.Eshift_dev ? *p.Eshift_dev : p.Eshift;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nwalk) return;
  const cplx old_ovlp = wp.ovlp[i];
  const cplx old_eloc = wp.pseudo_eloc[i];
  const cplx nov = new_ovlp[i];
  double scale = 1.0, dtheta = 0.0;
  if (!p.free_projection) {
    dtheta = nov.y - old_ovlp.y - mf[i].y;
    if (p.use_cp_constraint) scale = cos(dtheta) > 0.0 ? 1.0 : 0.0;
    else scale = fmax(0.0, cos(dtheta));
  }
  wp.theta[i] = mk(dtheta, 0.0);
  cplx eloc;
  if (p.hybrid) {
    cplx num = csub(csub(mf[i], hw[i]), csub(nov, old_ovlp));
    eloc = mk(num.x / p.dt + p.E0, num.y / p.dt);
  } else {
    eloc = cadd(cadd(E3[3 * i + 0], E3[3 * i + 1]), E3[3 * i + 2]);
  }
  cplx weight = wp.weight[i], phase = wp.phase[i];
  cplx wfac = mk(0.0, 0.0);
  if (!isfinite(eloc.x)) {
    weight = mk(0.0, 0.0);
    phase = mk(0.0, 0.0);
    eloc = old_eloc;
  } else {
    if (!p.free_projection) {
      const double hi = Eshift + p.upper_cutoff * sqrt(2.0 / p.dt);
      const double lo = Eshift - p.lower_cutoff * sqrt(2.0 / p.dt);
      if (stats) {
        atomicAdd(&stats[0], 1ull);
        if (eloc.x > hi) atomicAdd(&stats[1], 1ull);
        else if (eloc.x < lo) atomicAdd(&stats[2], 1ull);
      }
      eloc.x = fmin(fmax(eloc.x, lo), hi);
    }
    cplx eff = p.hybrid ? eloc : cscale(cadd(eloc, old_eloc), 0.5);
    cplx z = mk(-p.dt * (eff.x - Eshift), -p.dt * eff.y);
    cplx wf = cexp_(z);
    double aw = hypot(wf.x, wf.y);
    if (p.free_projection) weight = cmul(weight, cscale(wf, scale));
    else weight = cscale(weight, scale * aw);
    phase = cmul(phase, mk(wf.x / aw, wf.y / aw));
    if (fabs(scale) > 2.2250738585072014e-308) wfac = mk(wf.x / aw / scale, wf.y / aw / scale);
  }
  if (p.wfac) p.wfac[(p.wfac_pos ? (long)*p.wfac_pos : 0L) + (long)i * p.wfac_stride] = wfac;
  // bound_walker_weights
  const double a = hypot(weight.x, weight.y);
  if (stats) atomicAdd(&stats[3], 1ull);
  if (a > p.max_weight) {
    if (stats) atomicAdd(&stats[4], 1ull);
    weight = cscale(weight, p.max_weight / a);
  }
  wp.weight[i] = weight;
  wp.phase[i] = phase;
  wp.pseudo_eloc[i] = eloc;
  wp.ovlp[i] = nov;
  if (!p.hybrid) {
    wp.e1[i] = E3[3 * i + 0];
    wp.exx[i] = E3[3 * i + 1];
    wp.ej[i] = E3[3 * i + 2];
  }
}

// comb (population_control.hpp:34-65) + the single-rank slot plan of swap_walkers_async
// (:143-209).  One CTA; the cumulative sum is sequential so it rounds exactly like
// std::partial_sum, the teeth are placed in parallel by binary search (same comparisons as the
// sequential walk), and the copy plan is integer-only.
constexpr int PT = 1024;
__global__ void __launch_bounds__(PT) comb_kernel(WalkerProps wp, int nwalk, double r_in, unsigned long long seed,
                                                  unsigned long long call, int use_philox, PopWork pw,
                                                  const unsigned long long* call_dev) {
  __shared__ double s_total;
  __shared__ int s_last;
  __shared__ int s_ok;
  __shared__ double s_r;
  const int tid = threadIdx.x;
  for (int i = tid; i < nwalk; i += PT) pw.offspring[i] = 0;
  if (tid == 0) {
    double acc = 0.0;
    for (int i = 0; i < nwalk; ++i) {
      cplx w = wp.weight[i];
      acc = acc + hypot(w.x, w.y);
      pw.cum[i] = acc;
    }
    s_total = acc;
    s_ok = (acc > 1e-6) ? 1 : 0;
    int last = nwalk - 1;
    while (last > 0 && !(hypot(wp.weight[last].x, wp.weight[last].y) > 0.0)) --last;
    s_last = last;
    s_r = use_philox ? comb_uniform(seed, call_dev ? *call_dev : call) : r_in;
    *pw.flag = s_ok ? 0 : SFQ_ERR_WEIGHT_COLLAPSE;
  }
  __syncthreads();
  if (!s_ok) return;
  const double total = s_total, r = s_r;
  const int last = s_last;
  for (int ic = tid; ic < nwalk; ic += PT) {
    const double c = (double(ic) + r) * total / double(nwalk);
    int lo = 0, hi = nwalk;  // first j with c < cum[j]
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (c < pw.cum[mid]) hi = mid; else lo = mid + 1;
    }
    int iw = lo < last ? lo : last;
    atomicAdd(&pw.offspring[iw], 1);
  }
  __syncthreads();
  if (tid == 0) {
    // free slots ascending; copies fill them in ascending parent order
    int nfree = 0;
    for (int i = 0; i < nwalk; ++i)
      if (pw.offspring[i] == 0) pw.pairs[2 * (nfree++) + 1] = i;
    int nxt = 0;
    for (int i = 0; i < nwalk; ++i)
      for (int c = 1; c < pw.offspring[i]; ++c) pw.pairs[2 * (nxt++)] = i;
    *pw.npairs = nxt;
    if (nxt != nfree) *pw.flag = SFQ_ERR_INTERNAL;
  }
  __syncthreads();
  // every copy carries its parent's weight, so normalising first is the same as after
  for (int i = tid; i < nwalk; i += PT) {
    cplx w = wp.weight[i];
    double a = hypot(w.x, w.y);
    wp.weight[i] = mk(w.x / a, w.y / a);
  }
}

// comb over explicit |w| values (the bit-exact entry point sfq_comb)
__global__ void __launch_bounds__(PT) comb_weights_kernel(const double* wts, int nwalk, double r, int* offspring,
                                                          double* cum, int* flag) {
  __shared__ double s_total;
  __shared__ int s_last, s_ok;
  const int tid = threadIdx.x;
  for (int i = tid; i < nwalk; i += PT) offspring[i] = 0;
  if (tid == 0) {
    double acc = 0.0;
    for (int i = 0; i < nwalk; ++i) {
      acc = acc + wts[i];
      cum[i] = acc;
    }
    s_total = acc;
    s_ok = acc > 1e-6 ? 1 : 0;
    int last = nwalk - 1;
    while (last > 0 && wts[last] <= 0.0) --last;
    s_last = last;
    *flag = s_ok ? 0 : SFQ_ERR_WEIGHT_COLLAPSE;
  }
  __syncthreads();
  if (!s_ok) return;
  for (int ic = tid; ic < nwalk; ic += PT) {
    const double c = (double(ic) + r) * s_total / double(nwalk);
    int lo = 0, hi = nwalk;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (c < cum[mid]) hi = mid; else lo = mid + 1;
    }
    atomicAdd(&offspring[lo < s_last ? lo : s_last], 1);
  }
}

__global__ void copy_walkers_kernel(cplx* SM, long walker_elems, WalkerProps wp, const int* pairs, const int* npairs) {
  const int pidx = blockIdx.y;
  if (pidx >= *npairs) return;
  const int src = pairs[2 * pidx], dst = pairs[2 * pidx + 1];
  const cplx* s = SM + (long)src * walker_elems;
  cplx* d = SM + (long)dst * walker_elems;
  for (long e = blockIdx.x * blockDim.x + threadIdx.x; e < walker_elems; e += (long)gridDim.x * blockDim.x) d[e] = s[e];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    wp.weight[dst] = wp.weight[src];
    wp.phase[dst] = wp.phase[src];
    wp.pseudo_eloc[dst] = wp.pseudo_eloc[src];
    wp.e1[dst] = wp.e1[src];
    wp.exx[dst] = wp.exx[src];
    wp.ej[dst] = wp.ej[src];
    wp.ovlp[dst] = wp.ovlp[src];
    wp.theta[dst] = wp.theta[src];
  }
}

// E1 = E0 + scl * sum_aj G[w,a,j] haj[a,j]   (Real3IndexFactorization.hpp:157, :505-508)
__global__ void __launch_bounds__(RT) energy_e1_kernel(const cplx* G, const cplx* haj, cplx* E3, int nel, int nmo,
                                                       double E0, double scl, int addH1) {
  __shared__ cplx red[RT / 32];
  const int w = blockIdx.x;
  const long n = (long)nel * nmo;
  cplx acc = mk(0.0, 0.0);
  if (addH1)
    for (long e = threadIdx.x; e < n; e += RT) acc = cadd(acc, cmul(G[(long)w * n + e], haj[e]));
  cplx s = block_sum<RT>(acc, red);
  if (threadIdx.x == 0) {
    E3[3 * w + 0] = addH1 ? mk(E0 + scl * s.x, scl * s.y) : mk(0.0, 0.0);
    E3[3 * w + 1] = mk(0.0, 0.0);
    E3[3 * w + 2] = mk(0.0, 0.0);
  }
}

// one CTA per (n, w): exx[w, n0+n] = sum_ab T[w,a,n,b] T[w,b,n,a]; kl[w, n0+n] = sum_a T[w,a,n,a]
// nup < nel: COLLINEAR walkers, orbitals [0, nup) up and [nup, nel) down; the exchange pairs only
// orbitals of one spin (energy_impl runs per spin, Real3IndexFactorization.hpp:476-560)
__global__ void __launch_bounds__(RT) energy_exx_kernel(const cplx* T, int nel, int nv, int n0, int nchol,
                                                        cplx* exxn, cplx* kl, int nup) {
  __shared__ cplx red[RT / 32];
  const int n = blockIdx.x, w = blockIdx.y;
  const long rowstride = (long)nv * nel;  // T[(w*nel + a)][(n*nel + b)]
  const cplx* Tw = T + (long)w * nel * rowstride + (long)n * nel;
  cplx acc = mk(0.0, 0.0), tr = mk(0.0, 0.0);
  const int nn = nel * nel;
  for (int e = threadIdx.x; e < nn; e += RT) {
    const int a = e / nel, b = e % nel;
    const cplx tab = Tw[(long)a * rowstride + b];
    if (a == b) tr = cadd(tr, tab);
    if ((a < nup) != (b < nup)) continue;
    const cplx tba = Tw[(long)b * rowstride + a];
    acc = cadd(acc, cmul(tab, tba));
  }
  cplx s = block_sum<RT>(acc, red);
  cplx t = block_sum<RT>(tr, red);
  if (threadIdx.x == 0) {
    exxn[(long)w * nchol + n0 + n] = s;
    kl[(long)w * nchol + n0 + n] = t;
  }
}

// the same from the split-BF16 product: T planar in FP32, T[a][n][b] = (C[w*nel + a][n*nel + b],
// C[(W + w)*nel + a][n*nel + b]), sums in FP64
// nup < nel: COLLINEAR walkers, the exchange pairs orbitals of one spin only (as energy_exx_kernel)
__global__ void __launch_bounds__(RT) energy_exx_f32_kernel(const float* C, int W, int nel, int nv, int n0, int nchol,
                                                            long ldc, cplx* exxn, cplx* kl, int nup) {
  __shared__ cplx red[RT / 32];
  const int n = blockIdx.x, w = blockIdx.y;
  const float* Cr = C + (long)w * nel * ldc + (long)n * nel;
  const float* Ci = Cr + (long)W * nel * ldc;
  cplx acc = mk(0.0, 0.0), tr = mk(0.0, 0.0);
  const int nn = nel * nel;
  for (int e = threadIdx.x; e < nn; e += RT) {
    const int a = e / nel, b = e % nel;
    const cplx tab = mk(Cr[(long)a * ldc + b], Ci[(long)a * ldc + b]);
    if (a == b) tr = cadd(tr, tab);
    if ((a < nup) != (b < nup)) continue;
    const cplx tba = mk(Cr[(long)b * ldc + a], Ci[(long)b * ldc + a]);
    acc = cadd(acc, cmul(tab, tba));
  }
  cplx s = block_sum<RT>(acc, red);
  cplx t = block_sum<RT>(tr, red);
  if (threadIdx.x == 0) {
    exxn[(long)w * nchol + n0 + n] = s;
    kl[(long)w * nchol + n0 + n] = t;
  }
}

__global__ void __launch_bounds__(RT) energy_finish_kernel(const cplx* exxn, const cplx* kl, cplx* E3, int nchol,
                                                           double scl, int addEXX, int addEJ) {
  __shared__ cplx red[RT / 32];
  const int w = blockIdx.x;
  cplx a = mk(0.0, 0.0), b = mk(0.0, 0.0);
  for (int n = threadIdx.x; n < nchol; n += RT) {
    if (addEXX) a = cadd(a, exxn[(long)w * nchol + n]);
    if (addEJ) {
      cplx k = kl[(long)w * nchol + n];
      b = cadd(b, cmul(k, k));
    }
  }
  cplx sa = block_sum<RT>(a, red);
  cplx sb = block_sum<RT>(b, red);
  if (threadIdx.x == 0) {
    if (addEXX) E3[3 * w + 1] = cadd(E3[3 * w + 1], cscale(sa, -0.5 * scl));
    // CLOSED: 0.5 * 4 * sum Kl^2 (Real3IndexFactorization.hpp:169-173)
    if (addEJ) E3[3 * w + 2] = cadd(E3[3 * w + 2], cscale(sb, 0.5 * (scl == 2.0 ? 4.0 : 1.0)));
  }
}

template <typename E>
__global__ void permute_lnak_kernel(const E* tmp, E* Lnak, int nel, int nmo, int nchol) {
  // tmp[a][k][n] -> Lnak[n][a][k]
  const long total = (long)nel * nmo * nchol;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long n = e / ((long)nel * nmo);
    long r = e % ((long)nel * nmo);
    long a = r / nmo, k = r % nmo;
    Lnak[e] = tmp[(a * nmo + k) * nchol + n];
  }
}

__global__ void build_h1_kernel(const double* h, const double* v0, const cplx* vhs, double dt, double* H, int M) {
  const long total = (long)M * M;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long i = e / M, k = e % M;
    long t = k * M + i;
    double a = dt * h[e] + dt * v0[e] + vhs[e].x;
    double b = dt * h[t] + dt * v0[t] + vhs[t].x;
    // hermitize (real part): diagonal kept, off-diagonal averaged with the transpose
    double v = (i == k) ? a : 0.5 * a + 0.5 * b;
    H[e] = -0.5 * v;
  }
}

// add_one_body_shifts (one_body.hpp:64-82): H = dt (h + v0) + the mean-field shift's real part
__global__ void one_body_shift_kernel(const double* h, const double* v0, const cplx* vhs, double dt, double* H,
                                      long total) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x)
    H[e] = dt * h[e] + dt * v0[e] + vhs[e].x;
}

__global__ void add_identity_kernel(double* P, int M, double v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) P[(long)i * M + i] += v;
}

__global__ void threshold_kernel(double* P, long n, double drop) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    if (fabs(P[e]) < drop) P[e] = 0.0;
}

__global__ void real_of_kernel(const cplx* z, double* r, long n) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) r[e] = z[e].x;
}

__global__ void fill_kernel(cplx* p, long n, cplx v) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) p[e] = v;
}
__global__ void scale_kernel(cplx* p, long n, cplx s) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    p[e] = cmul(p[e], s);
}
__global__ void copy_kernel(cplx* d, const cplx* s, long n) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) d[e] = s[e];
}

__global__ void field_uniforms_kernel(double* out, unsigned long long seed, unsigned long long step, int nwalk,
                                      int nchol) {
  const int npair = (nchol + 1) / 2;
  const long total = (long)nwalk * npair;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int w = int(e / npair), j = int(e % npair);
    double u0, u1;
    field_uniform_pair(seed, step, (uint32_t)w, (uint32_t)j, u0, u1);
    out[(long)w * nchol + 2 * j] = u0;
    if (2 * j + 1 < nchol) out[(long)w * nchol + 2 * j + 1] = u1;
  }
}

inline int grid_for(long n) {
  long g = (n + 255) / 256;
  if (g > 148L * 32) g = 148L * 32;
  if (g < 1) g = 1;
  return int(g);
}

}  // namespace

int field_uniforms(double* out, unsigned long long seed, unsigned long long step, int nwalk, int nchol,
                   cudaStream_t st) {
  field_uniforms_kernel<<<grid_for((long)nwalk * ((nchol + 1) / 2)), 256, 0, st>>>(out, seed, step, nwalk, nchol);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int assemble_x(cplx* X, const double* vmf, cplx* hw, cplx* mf, const FieldParams& p, cudaStream_t st) {
  if (p.nwalk <= 0) return SFQ_OK;
  assemble_x_kernel<<<p.nwalk, RT, 0, st>>>(X, vmf, hw, mf, p);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int walker_update(const WalkerProps& w, const cplx* new_ovlp, const cplx* mf, const cplx* hw, const cplx* E3,
                  const UpdateParams& p, unsigned long long* stats, cudaStream_t st) {
  if (p.nwalk <= 0) return SFQ_OK;
  walker_update_kernel<<<(p.nwalk + 127) / 128, 128, 0, st>>>(w, new_ovlp, mf, hw, E3, p, stats);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

namespace {
__global__ void copy_rows_kernel(cplx* A, long elems, const int* pairs, const int* npairs) {
  const int pidx = blockIdx.y;
  if (pidx >= *npairs) return;
  const cplx* s = A + (long)pairs[2 * pidx] * elems;
  cplx* d = A + (long)pairs[2 * pidx + 1] * elems;
  for (long e = blockIdx.x * blockDim.x + threadIdx.x; e < elems; e += (long)gridDim.x * blockDim.x) d[e] = s[e];
}
}  // namespace

int copy_walker_rows(cplx* A, long elems, const PopWork& pw, int nwalk, cudaStream_t st) {
  if (nwalk <= 1 || elems <= 0) return SFQ_OK;
  int gx = int((elems + 255) / 256);
  if (gx > 8) gx = 8;
  copy_rows_kernel<<<dim3(gx, nwalk - 1), 256, 0, st>>>(A, elems, pw.pairs, pw.npairs);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

namespace {
// Slot lists travel in the kernel parameters, kSlotChunk at a time (no device allocation).
constexpr int kSlotChunk = 512;
struct SlotChunk {
  int v[2 * kSlotChunk];
};

// blockIdx.y: row within the chunk; DIR 0 packs walker -> row, 1 unpacks row -> walker
template <int DIR>
__global__ void walker_rows_kernel(cplx* SM, cplx* props, int nwalk, long elems, SlotChunk sl, int r0, cplx* rows) {
  const int r = blockIdx.y;
  const int w = sl.v[r];
  cplx* wr = SM + (long)w * elems;
  cplx* row = rows + (long)(r0 + r) * (elems + kWalkerProps);
  for (long e = blockIdx.x * blockDim.x + threadIdx.x; e < elems; e += (long)gridDim.x * blockDim.x) {
    if (DIR == 0) row[e] = wr[e];
    else wr[e] = row[e];
  }
  if (blockIdx.x == 0 && threadIdx.x < kWalkerProps) {
    if (DIR == 0) row[elems + threadIdx.x] = props[(long)threadIdx.x * nwalk + w];
    else props[(long)threadIdx.x * nwalk + w] = row[elems + threadIdx.x];
  }
}

__global__ void normalize_weights_kernel(cplx* weight, int nwalk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwalk) return;
  const cplx w = weight[i];
  const double a = hypot(w.x, w.y);
  weight[i] = mk(w.x / a, w.y / a);
}

__global__ void copy_pairs_kernel(cplx* SM, cplx* props, int nwalk, long elems, SlotChunk pr) {
  const int src = pr.v[2 * blockIdx.y], dst = pr.v[2 * blockIdx.y + 1];
  const cplx* s = SM + (long)src * elems;
  cplx* d = SM + (long)dst * elems;
  for (long e = blockIdx.x * blockDim.x + threadIdx.x; e < elems; e += (long)gridDim.x * blockDim.x) d[e] = s[e];
  if (blockIdx.x == 0 && threadIdx.x < kWalkerProps)
    props[(long)threadIdx.x * nwalk + dst] = props[(long)threadIdx.x * nwalk + src];
}

int row_grid_x(long elems) {
  long gx = (elems + 255) / 256;
  return int(gx < 1 ? 1 : (gx > 16 ? 16 : gx));
}

template <int DIR>
int walker_rows(cplx* SM, cplx* props, int nwalk, long elems, const int* slots, int n, cplx* rows, cudaStream_t st) {
  if (n < 0 || elems < 0) return SFQ_ERR_SHAPE;
  for (int r0 = 0; r0 < n; r0 += kSlotChunk) {
    const int m = n - r0 < kSlotChunk ? n - r0 : kSlotChunk;
    SlotChunk sl;
    for (int r = 0; r < m; ++r) {
      if (slots[r0 + r] < 0 || slots[r0 + r] >= nwalk) return SFQ_ERR_ARG;
      sl.v[r] = slots[r0 + r];
    }
    walker_rows_kernel<DIR><<<dim3(row_grid_x(elems), m), 256, 0, st>>>(SM, props, nwalk, elems, sl, r0, rows);
    SFQ_LAUNCHED();
  }
  return SFQ_OK;
}
}  // namespace

int pack_walker_rows(const cplx* SM, const cplx* props, int nwalk, long elems, const int* slots, int n, cplx* rows,
                     cudaStream_t st) {
  return walker_rows<0>(const_cast<cplx*>(SM), const_cast<cplx*>(props), nwalk, elems, slots, n, rows, st);
}

int unpack_walker_rows(cplx* SM, cplx* props, int nwalk, long elems, const int* slots, int n, const cplx* rows,
                       cudaStream_t st) {
  return walker_rows<1>(SM, props, nwalk, elems, slots, n, const_cast<cplx*>(rows), st);
}

int copy_walker_pairs(cplx* SM, cplx* props, int nwalk, long elems, const int* pairs, int n, int normalize,
                      cudaStream_t st) {
  if (n < 0 || elems < 0) return SFQ_ERR_SHAPE;
  std::vector<char> is_dst(size_t(nwalk > 0 ? nwalk : 0), 0);
  for (int k = 0; k < n; ++k) {
    const int s = pairs[2 * k], d = pairs[2 * k + 1];
    if (s < 0 || s >= nwalk || d < 0 || d >= nwalk || s == d || is_dst[d]) return SFQ_ERR_ARG;
    is_dst[d] = 1;
  }
  for (int k = 0; k < n; ++k)
    if (is_dst[pairs[2 * k]]) return SFQ_ERR_ARG;  // a source overwritten by another copy
  if (normalize && nwalk > 0) {
    normalize_weights_kernel<<<(nwalk + 255) / 256, 256, 0, st>>>(props, nwalk);  // WEIGHT is column 0
    SFQ_LAUNCHED();
  }
  for (int k0 = 0; k0 < n; k0 += kSlotChunk) {
    const int m = n - k0 < kSlotChunk ? n - k0 : kSlotChunk;
    SlotChunk pr;
    for (int k = 0; k < m; ++k) {
      pr.v[2 * k] = pairs[2 * (k0 + k)];
      pr.v[2 * k + 1] = pairs[2 * (k0 + k) + 1];
    }
    copy_pairs_kernel<<<dim3(row_grid_x(elems), m), 256, 0, st>>>(SM, props, nwalk, elems, pr);
    SFQ_LAUNCHED();
  }
  return SFQ_OK;
}

int population_control(cplx* SM, long walker_elems, const WalkerProps& w, int nwalk, double r_uniform,
                       unsigned long long seed, unsigned long long call, int use_philox, const PopWork& pw,
                       cudaStream_t st, const unsigned long long* call_dev) {
  if (nwalk <= 0) return SFQ_OK;
  comb_kernel<<<1, PT, 0, st>>>(w, nwalk, r_uniform, seed, call, use_philox, pw, call_dev);
  SFQ_LAUNCHED();
  int gx = int((walker_elems + 255) / 256);
  if (gx > 8) gx = 8;
  if (nwalk > 1) {
    dim3 grid(gx, nwalk - 1);
    copy_walkers_kernel<<<grid, 256, 0, st>>>(SM, walker_elems, w, pw.pairs, pw.npairs);
    SFQ_LAUNCHED();
  }
  return SFQ_OK;
}

int comb_weights(const double* wts, int nwalk, double r, int* offspring, double* cum, int* flag, cudaStream_t st) {
  if (nwalk <= 0) return SFQ_OK;
  comb_weights_kernel<<<1, PT, 0, st>>>(wts, nwalk, r, offspring, cum, flag);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int energy_e1(const cplx* G, const cplx* haj, cplx* E3, int nwalk, int nel, int nmo, double E0, double scl,
              int addH1, cudaStream_t st) {
  if (nwalk <= 0) return SFQ_OK;
  energy_e1_kernel<<<nwalk, RT, 0, st>>>(G, haj, E3, nel, nmo, E0, scl, addH1);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int energy_exx_reduce(const cplx* T, int nwalk, int nel, int nv, int n0, int nchol, cplx* exxn, cplx* kl,
                      cudaStream_t st, int nup) {
  if (nwalk <= 0 || nv <= 0) return SFQ_OK;
  dim3 grid(nv, nwalk);
  energy_exx_kernel<<<grid, RT, 0, st>>>(T, nel, nv, n0, nchol, exxn, kl, nup < 0 ? nel : nup);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int energy_exx_reduce_f32(const float* C, int nwalk, int nel, int nv, int n0, int nchol, long ldc, cplx* exxn,
                          cplx* kl, cudaStream_t st, int nup) {
  if (nwalk <= 0 || nv <= 0) return SFQ_OK;
  dim3 grid(nv, nwalk);
  energy_exx_f32_kernel<<<grid, RT, 0, st>>>(C, nwalk, nel, nv, n0, nchol, ldc, exxn, kl, nup < 0 ? nel : nup);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int energy_finish(const cplx* exxn, const cplx* kl, cplx* E3, int nwalk, int nchol, double scl, int addEXX,
                  int addEJ, cudaStream_t st) {
  if (nwalk <= 0) return SFQ_OK;
  energy_finish_kernel<<<nwalk, RT, 0, st>>>(exxn, kl, E3, nchol, scl, addEXX, addEJ);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

namespace {
__global__ void copy_where_kernel(cplx* dst, const cplx* src, const int* mask, int want, long n) {
  const long w = blockIdx.y;
  if ((mask[w] != 0) != (want != 0)) return;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    dst[w * n + e] = src[w * n + e];
}

__global__ void check_symmetric_kernel(const double* L, int M, int Nc, int* flag) {
  const long total = (long)M * M * Nc;
  int bad = 0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long row = t / Nc, n = t % Nc;
    const long i = row / M, k = row % M;
    if (i < k) {
      const long long a = __double_as_longlong(L[t]);
      const long long b = __double_as_longlong(L[(k * M + i) * Nc + n]);
      bad |= (a != b);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

__global__ void pack_upper_kernel(const double* L, int M, int Nc, double* Lp) {
  const long total = (long)M * M * Nc;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long row = t / Nc, n = t % Nc;
    const long i = row / M, k = row % M;
    if (i <= k) Lp[upper_index(i, k, M) * Nc + n] = L[t];
  }
}

__global__ void unpack_symmetric_kernel(const cplx* Vp, int W, int M, cplx* V) {
  const long MM = (long)M * M, P = (long)M * (M + 1) / 2;
  const long total = (long)W * MM;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long w = t / MM, r = t % MM;
    const long i = r / M, k = r % M;
    V[t] = Vp[w * P + (i <= k ? upper_index(i, k, M) : upper_index(k, i, M))];
  }
}
}  // namespace

int copy_walkers_where(cplx* dst, const cplx* src, const int* mask, int want, int W, long n, cudaStream_t st) {
  dim3 grid(unsigned((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), unsigned(W));
  copy_where_kernel<<<grid, 256, 0, st>>>(dst, src, mask, want, n);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int check_symmetric(const double* L, int M, int Nc, int* flag, cudaStream_t st) {
  check_symmetric_kernel<<<grid_for((long)M * M * Nc), 256, 0, st>>>(L, M, Nc, flag);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int pack_upper(const double* L, int M, int Nc, double* Lp, cudaStream_t st) {
  pack_upper_kernel<<<grid_for((long)M * M * Nc), 256, 0, st>>>(L, M, Nc, Lp);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int unpack_symmetric(const cplx* Vp, int W, int M, cplx* V, cudaStream_t st) {
  unpack_symmetric_kernel<<<grid_for((long)W * M * M), 256, 0, st>>>(Vp, W, M, V);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int permute_lnak(const void* tmp, void* Lnak, int nel, int nmo, int nchol, int esz, cudaStream_t st) {
  const int g = grid_for((long)nel * nmo * nchol);
  if (esz == 16)
    permute_lnak_kernel<cplx><<<g, 256, 0, st>>>((const cplx*)tmp, (cplx*)Lnak, nel, nmo, nchol);
  else
    permute_lnak_kernel<double><<<g, 256, 0, st>>>((const double*)tmp, (double*)Lnak, nel, nmo, nchol);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int build_h1(const double* h, const double* v0, const cplx* vhs, double dt, double* H, int nmo, cudaStream_t st) {
  build_h1_kernel<<<grid_for((long)nmo * nmo), 256, 0, st>>>(h, v0, vhs, dt, H, nmo);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int one_body_shift(const double* h, const double* v0, const cplx* vhs, double dt, double* H, int nmo,
                   cudaStream_t st) {
  one_body_shift_kernel<<<grid_for((long)nmo * nmo), 256, 0, st>>>(h, v0, vhs, dt, H, (long)nmo * nmo);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int add_identity(double* P, int nmo, double v, cudaStream_t st) {
  add_identity_kernel<<<(nmo + 255) / 256, 256, 0, st>>>(P, nmo, v);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int threshold_real(double* P, long n, double drop, cudaStream_t st) {
  threshold_kernel<<<grid_for(n), 256, 0, st>>>(P, n, drop);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int real_of(const cplx* z, double* r, long n, cudaStream_t st) {
  real_of_kernel<<<grid_for(n), 256, 0, st>>>(z, r, n);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int fill_cplx(cplx* p, long n, cplx v, cudaStream_t st) {
  if (n <= 0) return SFQ_OK;
  fill_kernel<<<grid_for(n), 256, 0, st>>>(p, n, v);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int scale_cplx(cplx* p, long n, cplx s, cudaStream_t st) {
  if (n <= 0) return SFQ_OK;
  scale_kernel<<<grid_for(n), 256, 0, st>>>(p, n, s);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int copy_walkers_prop(cplx* dst, const cplx* src, long n, cudaStream_t st) {
  if (n <= 0) return SFQ_OK;
  copy_kernel<<<grid_for(n), 256, 0, st>>>(dst, src, n);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace sfq
