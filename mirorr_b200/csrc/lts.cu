// lts.cu -- the least-trimmed-squares fit on the device.
//
// One cooperative launch runs the whole inner loop of OptimizeTransform
// (classic: itkMirorrRegistrationMethod.txx:785-999; symmetric:
// itkSymMirorrRegistrationMethod.txx:771-1442).  Per inner iteration:
//   residuals r_i (FP64) under the current final transform(s);
//   the threshold r_nth: the maximum on the first iteration, otherwise the
//     exact value of rank min(floor(f N), N-1) by an MSD radix select on the
//     residual bit patterns (grid-wide histograms until at most one CTA's
//     worth of keys share the prefix, then those keys ranked by counting);
//   subset {r_i <= r_nth}: count, first and second moments of the
//     (initial, moved) pairs about the first pair in one sweep, reduced per
//     CTA and summed in a fixed order (deterministic), then centred;
//   the FP64 solve (affine normal equations / Horn quaternion, symmetric
//     half-space algebra) in one thread, and the loop test.
// CTAs meet at a software grid barrier whose wait is bounded (about one
// second); a timeout raises an error flag and every CTA returns.
#include <cooperative_groups.h>

#include <mutex>

#include "gridsel.cuh"
#include "kernels.cuh"

namespace mb2 {

namespace {

constexpr int kThreads = 256;
constexpr int kBins = 4096;
constexpr int kCandMax = kThreads;  // keys left for the final rank (one per thread)
constexpr int kPartial = 32;  // doubles per CTA partial
// Polls of a grid-barrier wait (about 0.84 s with the 100 ns back-off) before
// the wait gives up, raises the error flag and every CTA returns.
constexpr long long kDefaultSpinLimit = 1LL << 23;

struct LtsCtl {
  unsigned int bar_count;
  unsigned int bar_gen;
  int err;
  int pad;
  unsigned long long maxkey;
  unsigned long long ncand;
};

struct LtsArgs {
  LtsState *state;
  const double *init;
  const double *moved;
  const long long *n_dev;
  double *resid;
  double *partial;        // gridDim.x * kPartial
  unsigned int *hist;     // 3 * kBins
  unsigned long long *cand;
  LtsCtl *ctl;
  long long spin_limit;   // polls of a grid-barrier wait before it gives up
};

__device__ inline bool grid_sync(LtsCtl *ctl, long long spin_limit, unsigned int nctas) {
  return grid_barrier(&ctl->bar_count, &ctl->bar_gen, &ctl->err, spin_limit, nctas);
}

__device__ inline void load_cg(void *dst, const void *src, int bytes) {
  const unsigned long long *s = static_cast<const unsigned long long *>(src);
  unsigned long long *d = static_cast<unsigned long long *>(dst);
  for (int i = threadIdx.x; i < bytes / 8; i += blockDim.x) d[i] = __ldcg(s + i);
}

// Sums each of v[0, N) over the CTA (per value: shuffle tree within each
// warp, then the warps in order); out[q] in shared memory, valid for every
// thread on return.
template <int N>
__device__ inline void block_sums(const double (&v)[N], double *red /* N * 32 */, double *out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) red[q * 32 + wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double r = 0.0;
    for (int w = 0; w < nw; ++w) r += red[threadIdx.x * 32 + w];
    out[threadIdx.x] = r;
  }
  __syncthreads();
}

// out[q] = sum over the grid's CTAs b of part[b * kPartial + q0 + q], q < nq:
// warp q % nwarps takes value q, its lanes stride over b, then a shuffle tree
// (a fixed order).  out in shared memory, valid for every thread on return.
__device__ inline void grid_partial_sums(const double *part, int q0, int nq, double *out,
                                         int nctas) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = wid; q < nq; q += nw) {
    double x = 0.0;
    for (int b = lane; b < nctas; b += 32) x += __ldcg(&part[(long long)b * kPartial + q0 + q]);
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) out[q] = x;
  }
  __syncthreads();
}

__device__ inline double residual(const LtsState &s, const double *x, const double *y) {
  double p[3], q[3];
  tfm_apply(s.fin, x, p);
  if (s.symmetric) {
    tfm_apply(s.finb, y, q);
  } else {
    q[0] = y[0]; q[1] = y[1]; q[2] = y[2];
  }
  double r = 0.0;
  for (int i = 0; i < 3; ++i) {
    double d = p[i] - q[i];
    r += d * d;
  }
  return r;
}

// The LTS loop run by `ncta` CTAs (index `cta` among them) that meet at the
// bounded grid barrier of a.ctl.
__device__ void lts_body(const LtsArgs &a, int cta, int ncta) {
  __shared__ __align__(16) LtsState s;
  __shared__ unsigned int h[kBins];
  __shared__ unsigned long long ck[kCandMax];
  __shared__ double red_n[28 * 32];
  __shared__ double s_nth;
  __shared__ unsigned long long s_key;
  __shared__ unsigned long long s_pair[2];
  const long long n = __ldcg(&a.n_dev[0]) + __ldcg(&a.n_dev[1]);
  const long long gstride = (long long)ncta * blockDim.x;
  const long long gtid = (long long)cta * blockDim.x + threadIdx.x;

  for (int guard = 0; guard < 200; ++guard) {
    load_cg(&s, a.state, sizeof(LtsState));
    __syncthreads();
    if (!s.running || n <= 0) break;
    const bool first = s.fraction > 0.99999;
    // ---- residuals (+ max or first histogram) ----------------------------
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
    if (cta == 0)
      for (int i = threadIdx.x; i < kBins; i += blockDim.x) {
        a.hist[kBins + i] = 0;  // next two passes' buffers
      }
    __syncthreads();
    unsigned long long kmax = 0;
    for (long long i = gtid; i < n; i += gstride) {
      double r = residual(s, a.init + 3 * i, a.moved + 3 * i);
      a.resid[i] = r;
      unsigned long long key = (unsigned long long)__double_as_longlong(r);
      if (first) {
        if (key > kmax) kmax = key;
      } else {
        hist_add(h, (unsigned)(key >> 52) & (kBins - 1));
      }
    }
    if (first) {
      for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_down_sync(0xffffffffu, kmax, off);
        if (o > kmax) kmax = o;
      }
      if ((threadIdx.x & 31) == 0 && kmax) atomicMax(&a.ctl->maxkey, kmax);
    } else {
      __syncthreads();
      for (int i = threadIdx.x; i < kBins; i += blockDim.x)
        if (h[i]) atomicAdd(&a.hist[i], h[i]);
    }
    if (!grid_sync(a.ctl, a.spin_limit, (unsigned)ncta)) return;
    double nth;
    if (first) {
      if (threadIdx.x == 0) s_key = __ldcg(&a.ctl->maxkey);
      __syncthreads();
      nth = __longlong_as_double((long long)s_key);
    } else {
      // ---- radix select of rank k -----------------------------------------
      unsigned long long k = (unsigned long long)(unsigned int)(s.fraction * (double)n);
      if (k > (unsigned long long)(n - 1)) k = n - 1;
      unsigned long long prefix = 0, mask = 0;
      int shift = 52, bits = 12, pass = 0;
      unsigned long long bucket = 0;
      while (true) {
        // every CTA scans the global histogram of this pass identically
        const unsigned int *gh = a.hist + (pass % 3) * kBins;
        __syncthreads();
        for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = __ldcg(&gh[i]);
        __syncthreads();
        int d = 0;
        unsigned long long cum = 0;
        find_bucket<kBins, kThreads>(h, k, 1 << bits, s_pair, &d, &cum);
        bucket = h[d];
        k -= cum;
        prefix |= (unsigned long long)d << shift;
        mask |= ((1ULL << bits) - 1ULL) << shift;
        __syncthreads();
        if (bucket <= (unsigned long long)kCandMax || shift == 0) break;
        // more than one CTA's worth of keys share the prefix: refine it
        // next pass
        ++pass;
        bits = shift >= 12 ? 12 : shift;
        shift -= bits;
        if (cta == 0) {
          unsigned int *zb = a.hist + ((pass + 1) % 3) * kBins;
          for (int i = threadIdx.x; i < kBins; i += blockDim.x) zb[i] = 0;
        }
        for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
        __syncthreads();
        for (long long i = gtid; i < n; i += gstride) {
          unsigned long long key = (unsigned long long)__double_as_longlong(a.resid[i]);
          if ((key & mask) == prefix) hist_add(h, (unsigned)(key >> shift) & ((1u << bits) - 1u));
        }
        __syncthreads();
        unsigned int *gh2 = a.hist + (pass % 3) * kBins;
        for (int i = threadIdx.x; i < kBins; i += blockDim.x)
          if (h[i]) atomicAdd(&gh2[i], h[i]);
        if (!grid_sync(a.ctl, a.spin_limit, (unsigned)ncta)) return;
      }
      if (shift == 0) {
        // every bit fixed: the bucket's keys all equal the prefix
        nth = __longlong_as_double((long long)prefix);
      } else {
        // ---- gather the bucket's keys (at most one per thread) and rank them
        for (long long i = gtid; i < n; i += gstride) {
          unsigned long long key = (unsigned long long)__double_as_longlong(a.resid[i]);
          if ((key & mask) == prefix) {
            unsigned long long pos = atomicAdd(&a.ctl->ncand, 1ULL);
            if (pos < (unsigned long long)kCandMax) a.cand[pos] = key;
          }
        }
        if (!grid_sync(a.ctl, a.spin_limit, (unsigned)ncta)) return;
        if (threadIdx.x == 0) s_key = __ldcg(&a.ctl->ncand);
        __syncthreads();
        const int nc = (int)(s_key < (unsigned long long)kCandMax ? s_key : kCandMax);
        const unsigned long long kk = k < (unsigned long long)nc ? k : (nc > 0 ? nc - 1 : 0);
        // rank by counting: key i has rank kk iff lo_i <= kk < lo_i + eq_i
        for (int i = threadIdx.x; i < nc; i += blockDim.x) ck[i] = __ldcg(&a.cand[i]);
        __syncthreads();
        if (threadIdx.x < nc) {
          const unsigned long long v = ck[threadIdx.x];
          int lo = 0, eq = 0;
          for (int j = 0; j < nc; ++j) {
            const unsigned long long u = ck[j];
            lo += u < v;
            eq += u == v;
          }
          if ((unsigned long long)lo <= kk && kk < (unsigned long long)(lo + eq))
            s_nth = __longlong_as_double((long long)v);
        }
        __syncthreads();
        nth = s_nth;
      }
    }
    // ---- subset moments in one sweep: count, first and second moments of
    // the pairs z = (initial, moved) about the first pair z0 (near the data,
    // so centring afterwards loses nothing in FP64) ------------------------
    double z0[6];
    for (int c = 0; c < 3; ++c) {
      z0[c] = __ldg(&a.init[c]);
      z0[3 + c] = __ldg(&a.moved[c]);
    }
    double acc[28];
#pragma unroll
    for (int q = 0; q < 28; ++q) acc[q] = 0.0;
    for (long long i = gtid; i < n; i += gstride) {
      if (a.resid[i] <= nth) {
        double z[6];
        for (int c = 0; c < 3; ++c) {
          z[c] = a.init[3 * i + c] - z0[c];
          z[3 + c] = a.moved[3 * i + c] - z0[3 + c];
        }
        acc[0] += 1.0;
#pragma unroll
        for (int r = 0; r < 6; ++r) acc[1 + r] += z[r];
        int q = 7;
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
          for (int c = r; c < 6; ++c) acc[q++] += z[r] * z[c];
      }
    }
    __shared__ double s_out[28];
    block_sums<28>(acc, red_n, s_out);
    if (threadIdx.x < 28) a.partial[(long long)cta * kPartial + threadIdx.x] = s_out[threadIdx.x];
    if (!grid_sync(a.ctl, a.spin_limit, (unsigned)ncta)) return;
    if (cta == 0) grid_partial_sums(a.partial, 0, 28, s_out, ncta);
    // the solve: warp 0 of CTA 0; the symmetric fit's two square roots run
    // on lanes 0 and 1 at once
    __shared__ SymHalf s_half;
    __shared__ double s_root[2][16];
    if (cta == 0 && threadIdx.x < 32) {
      if (threadIdx.x == 0) {
        LtsMoments mo;
        const double cnt = s_out[0];
        double m[6];
        for (int r = 0; r < 6; ++r) m[r] = s_out[1 + r] / cnt;
        mo.n = cnt;
        for (int c = 0; c < 3; ++c) { mo.mean_i[c] = z0[c] + m[c]; mo.mean_m[c] = z0[3 + c] + m[3 + c]; }
        int q = 7;
        for (int r = 0; r < 6; ++r)
          for (int c = r; c < 6; ++c) {
            const double zz = s_out[q++] - cnt * m[r] * m[c];
            mo.Z[6 * r + c] = zz;
            mo.Z[6 * c + r] = zz;
          }
        if (s.symmetric) lts_symmetric_pre(s, mo, s_half);
        else lts_classic_step(s, mo);
      }
      __syncwarp();
      if (s.symmetric && threadIdx.x < 2)
        half_step(s_half.K[threadIdx.x], s_half.t[threadIdx.x], s_root[threadIdx.x]);
      __syncwarp();
      if (threadIdx.x == 0) {
        if (s.symmetric) lts_symmetric_post(s, s_half, s_root[0], s_root[1]);
        s.fraction = s.lts_keep;
        s.iter += 1;
        s.running = lts_continue(s) ? 1 : 0;
        if (s.iter > 101) s.running = 0;
        // reset select scratch for the next iteration
        a.ctl->maxkey = 0;
        a.ctl->ncand = 0;
        *a.state = s;
        __threadfence();
      }
    }
    if (cta == 0) {
      __syncthreads();
      for (int i = threadIdx.x; i < kBins; i += blockDim.x) a.hist[i] = 0;
    }
    if (!grid_sync(a.ctl, a.spin_limit, (unsigned)ncta)) return;
  }
}

__global__ void __launch_bounds__(kThreads) lts_kernel(LtsArgs a) {
  lts_body(a, blockIdx.x, gridDim.x);
}

// Several independent fits in one cooperative launch: fit f runs on CTAs
// [f ncta, (f + 1) ncta) with its own arguments and barrier.
__global__ void __launch_bounds__(kThreads) lts_batch_kernel(const LtsArgs *args, int ncta) {
  const LtsArgs a = args[blockIdx.x / ncta];
  lts_body(a, blockIdx.x % ncta, ncta);
}

// Zeroes each fit's barrier, select control and histograms (CTA f: fit f) so
// a batch's launch sequence has the same nodes whatever the number of fits.
__global__ void lts_batch_zero_kernel(const LtsArgs *args, unsigned long long words) {
  uint4 *p = reinterpret_cast<uint4 *>(args[blockIdx.x].ctl);
  for (unsigned long long i = threadIdx.x; i < words; i += blockDim.x) p[i] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace

mirorr_status lts_run(LtsWork &w, LtsState &hs, const double *init_dev, const double *moved_dev,
                      const long long *n_dev, long long n, cudaStream_t st, int *inner_iters,
                      long long *n_used, const unsigned int *watch_dev,
                      unsigned int *watch_host) {
  if (watch_host) *watch_host = 0;
  lts_begin(hs);
  if (n <= 0) {
    lts_finish(hs);
    if (inner_iters) *inner_iters = 0;
    if (n_used) *n_used = 0;
    return MIRORR_OK;
  }
  MB2_TRY(lts_issue(w, &hs, init_dev, moved_dev, n_dev, n, st, nullptr, watch_dev));
  MB2_CUDA_TRY(cudaStreamSynchronize(st));
  return lts_collect(w, nullptr, hs, inner_iters, n_used, watch_host);
}

// What lts_issue reads back, in host memory (pinned staging for a captured
// sequence, or the work area's own copy).
struct LtsOut {
  LtsState state;
  LtsCtl ctl;
  long long n[2];
  unsigned int watch;
};

size_t lts_out_bytes() { return sizeof(LtsOut); }

mirorr_status lts_issue(LtsWork &w, const LtsState *state_in, const double *init_dev,
                        const double *moved_dev, const long long *n_dev, long long n,
                        cudaStream_t st, void *out_host, const unsigned int *watch_dev) {
  int dev = 0;
  MB2_CUDA_TRY(cudaGetDevice(&dev));
  if (w.max_ctas == 0) {
    int sms = 0, per = 0, coop = 0;
    MB2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MB2_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) {
      set_error("device does not support cooperative launches");
      return MIRORR_ECUDA;
    }
    MB2_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, lts_kernel, kThreads, 0));
    if (per < 1) {
      set_error("LTS kernel cannot be resident");
      return MIRORR_ECUDA;
    }
    w.max_ctas = sms * (per > 1 ? 1 : per);
  }
  long long want = (n + 4 * kThreads - 1) / (4 * kThreads);
  int grid = (int)(want < 1 ? 1 : (want > w.max_ctas ? w.max_ctas : want));
  MB2_TRY(w.state.ensure(sizeof(LtsState)));
  MB2_TRY(w.resid.ensure(sizeof(double) * n));
  MB2_TRY(w.partial.ensure(sizeof(double) * kPartial * (size_t)grid));
  MB2_TRY(w.hist.ensure(sizeof(unsigned int) * 3 * kBins));
  MB2_TRY(w.ctrl.ensure(sizeof(LtsCtl)));
  MB2_TRY(w.cand.ensure(sizeof(unsigned long long) * kCandMax));
  if (!out_host) {
    MB2_TRY(w.out.ensure(sizeof(LtsOut)));
    out_host = w.out.ptr;
  }
  LtsOut *o = static_cast<LtsOut *>(out_host);
  MB2_CUDA_TRY(cudaMemcpyAsync(w.state.ptr, state_in, sizeof(LtsState), cudaMemcpyHostToDevice, st));
  MB2_CUDA_TRY(cudaMemsetAsync(w.hist.ptr, 0, sizeof(unsigned int) * 3 * kBins, st));
  MB2_CUDA_TRY(cudaMemsetAsync(w.ctrl.ptr, 0, sizeof(LtsCtl), st));
  LtsArgs a;
  a.state = w.state.as<LtsState>();
  a.init = init_dev;
  a.moved = moved_dev;
  a.n_dev = n_dev;
  a.resid = w.resid.as<double>();
  a.partial = w.partial.as<double>();
  a.hist = w.hist.as<unsigned int>();
  a.cand = w.cand.as<unsigned long long>();
  a.ctl = w.ctrl.as<LtsCtl>();
  a.spin_limit = w.spin_limit > 0 ? w.spin_limit : kDefaultSpinLimit;
  void *args[] = {&a};
  MB2_CUDA_TRY(cudaLaunchCooperativeKernel((void *)lts_kernel, dim3(grid), dim3(kThreads), args, 0, st));
  ++g_launches;
  MB2_CUDA_TRY(cudaMemcpyAsync(&o->state, w.state.ptr, sizeof(LtsState), cudaMemcpyDeviceToHost, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(&o->ctl, w.ctrl.ptr, sizeof(LtsCtl), cudaMemcpyDeviceToHost, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(o->n, n_dev, sizeof(o->n), cudaMemcpyDeviceToHost, st));
  if (watch_dev)
    MB2_CUDA_TRY(cudaMemcpyAsync(&o->watch, watch_dev, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  else
    o->watch = 0;
  return MIRORR_OK;
}

mirorr_status lts_collect(LtsWork &w, const void *out_host, LtsState &hs, int *inner_iters,
                          long long *n_used, unsigned int *watch_host) {
  const LtsOut *o = static_cast<const LtsOut *>(out_host ? out_host : w.out.ptr);
  hs = o->state;
  if (watch_host) *watch_host = o->watch;
  if (n_used) *n_used = o->n[0] + o->n[1];
  if (o->ctl.err) {
    set_error("LTS grid barrier timed out");
    return MIRORR_ETIMEOUT;
  }
  if (inner_iters) *inner_iters = hs.iter;
  lts_finish(hs);
  return MIRORR_OK;
}

// ---- many fits in one cooperative launch ----------------------------------------
//
// Fit f's CTAs meet at their own barrier (its LtsCtl); each fit has its own
// state, counters and scratch (LtsFit, all device pointers).  The caller has
// run lts_begin on every state it uploaded and runs lts_finish on each after
// reading it back.  A fit whose state is not running returns at once.
size_t lts_args_bytes() { return sizeof(LtsArgs); }

size_t lts_fit_scratch_bytes(long long n_max, int ncta) {
  const size_t a = 256;
  auto up = [&](size_t v) { return (v + a - 1) / a * a; };
  return up(sizeof(LtsCtl)) + up(sizeof(unsigned int) * 3 * kBins) +
         up(sizeof(unsigned long long) * kCandMax) + up(sizeof(double) * kPartial * (size_t)ncta) +
         up(sizeof(double) * (size_t)(n_max > 0 ? n_max : 1));
}

mirorr_status lts_batch_launch(const LtsFit *fits, int nfits, int ncta, long long spin_limit,
                               DevBuf &args_dev, HostBuf &args_host, cudaStream_t st) {
  if (nfits <= 0) return MIRORR_OK;
  int dev = 0, sms = 0, per = 0;
  MB2_CUDA_TRY(cudaGetDevice(&dev));
  MB2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MB2_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, lts_batch_kernel, kThreads, 0));
  if ((long long)nfits * ncta > (long long)sms * per) {
    set_error("%d fits of %d CTAs exceed the %d co-resident CTAs of the LTS kernel", nfits, ncta,
              sms * per);
    return MIRORR_EINVAL;
  }
  MB2_TRY(args_dev.ensure(sizeof(LtsArgs) * nfits));
  MB2_TRY(args_host.ensure(sizeof(LtsArgs) * nfits));
  LtsArgs *ha = args_host.as<LtsArgs>();
  const size_t al = 256;
  auto up = [&](size_t v) { return (v + al - 1) / al * al; };
  for (int f = 0; f < nfits; ++f) {
    unsigned char *p = static_cast<unsigned char *>(fits[f].scratch);
    LtsArgs &a = ha[f];
    a.state = fits[f].state;
    a.init = fits[f].init;
    a.moved = fits[f].moved;
    a.n_dev = fits[f].n_dev;
    a.ctl = reinterpret_cast<LtsCtl *>(p);
    p += up(sizeof(LtsCtl));
    a.hist = reinterpret_cast<unsigned int *>(p);
    p += up(sizeof(unsigned int) * 3 * kBins);
    a.cand = reinterpret_cast<unsigned long long *>(p);
    p += up(sizeof(unsigned long long) * kCandMax);
    a.partial = reinterpret_cast<double *>(p);
    p += up(sizeof(double) * kPartial * (size_t)ncta);
    a.resid = reinterpret_cast<double *>(p);
    a.spin_limit = spin_limit > 0 ? spin_limit : kDefaultSpinLimit;
  }
  MB2_CUDA_TRY(cudaMemcpyAsync(args_dev.ptr, ha, sizeof(LtsArgs) * nfits, cudaMemcpyHostToDevice, st));
  const LtsArgs *dargs = args_dev.as<LtsArgs>();
  // zeroed barrier, select control and histograms of every fit (the scratch
  // starts 256-byte aligned: the region is whole 16-byte words)
  const size_t zbytes = up(sizeof(LtsCtl)) + up(sizeof(unsigned int) * 3 * kBins);
  lts_batch_zero_kernel<<<nfits, 256, 0, st>>>(dargs, (unsigned long long)(zbytes / 16));
  MB2_LAUNCH_CHECK();
  ++g_launches;
  void *kargs[] = {(void *)&dargs, (void *)&ncta};
  MB2_CUDA_TRY(cudaLaunchCooperativeKernel((void *)lts_batch_kernel, dim3(nfits * ncta),
                                           dim3(kThreads), kargs, 0, st));
  ++g_launches;
  return MIRORR_OK;
}

// Error flag of fit f's barrier (device word of its scratch).
const int *lts_fit_error_flag(const void *scratch) {
  return &static_cast<const LtsCtl *>(scratch)->err;
}

// ---- allocation-free variant ----------------------------------------------------
//
// lts_run_noalloc runs the same kernel with the same grid as lts_run, but every
// scratch buffer lives in one static device array, so the call allocates no
// device memory.  Its address is looked up once per device (the first call on
// that device) with cudaGetSymbolAddress.  Layout, in bytes:
//   [0, 4096)        LtsState (uploaded each call)
//   [4096, 4352)     LtsCtl (zeroed each call)
//   [4352, 4608)     point-pair counters {n, 0} (uploaded each call)
//   [4608, +48 KB)   3 radix histograms of 4096 bins (zeroed each call)
//   then             256 candidate keys, kNaMaxCtas * 32 partial sums,
//                    MIRORR_LTS_NOALLOC_MAX_POINTS residuals.
// Two calls in flight on one device share the array and race.

namespace {

constexpr int kNaMaxCtas = 256;
constexpr int kNaMaxDevices = 64;
constexpr size_t kNaState = 0;
constexpr size_t kNaCtl = 4096;
constexpr size_t kNaCount = kNaCtl + 256;
constexpr size_t kNaHist = kNaCount + 256;
constexpr size_t kNaCand = kNaHist + sizeof(unsigned int) * 3 * kBins;
constexpr size_t kNaPartial = kNaCand + sizeof(unsigned long long) * kCandMax;
constexpr size_t kNaResid = kNaPartial + sizeof(double) * kPartial * kNaMaxCtas;
constexpr size_t kNaBytes = kNaResid + sizeof(double) * (size_t)MIRORR_LTS_NOALLOC_MAX_POINTS;
static_assert(sizeof(LtsState) <= kNaCtl - kNaState, "LtsState slot");
static_assert(sizeof(LtsCtl) <= kNaCount - kNaCtl, "LtsCtl slot");
static_assert(kNaHist % 256 == 0 && kNaCand % 256 == 0 && kNaPartial % 256 == 0 &&
                  kNaResid % 256 == 0, "slot alignment");

static __device__ __align__(256) unsigned char g_lts_scratch[kNaBytes];

std::mutex g_na_mu;
unsigned char *g_na_ptr[kNaMaxDevices];
int g_na_ctas[kNaMaxDevices];

// One-time set-up per device (the calling thread's current device): the
// scratch address and the co-resident CTA count of the cooperative launch.
mirorr_status na_setup(int dev, unsigned char **ptr, int *ctas) {
  std::lock_guard<std::mutex> lock(g_na_mu);
  if (dev < 0 || dev >= kNaMaxDevices) {
    set_error("device ordinal %d is beyond the %d devices the no-allocation LTS supports", dev,
              kNaMaxDevices);
    return MIRORR_ERANGE;
  }
  if (!g_na_ptr[dev]) {
    int sms = 0, per = 0, coop = 0;
    MB2_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MB2_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) {
      set_error("device does not support cooperative launches");
      return MIRORR_ECUDA;
    }
    MB2_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, lts_kernel, kThreads, 0));
    if (per < 1) {
      set_error("LTS kernel cannot be resident");
      return MIRORR_ECUDA;
    }
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_lts_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress of the LTS scratch array failed on device %d: %s", dev,
                cudaGetErrorString(e));
      return MIRORR_ECUDA;
    }
    g_na_ctas[dev] = sms * (per > 1 ? 1 : per);
    g_na_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *ptr = g_na_ptr[dev];
  *ctas = g_na_ctas[dev];
  return MIRORR_OK;
}

}  // namespace

mirorr_status lts_run_noalloc(LtsState &hs, const double *init_dev, const double *moved_dev,
                              long long n, cudaStream_t st, int *inner_iters) {
  if (n > (long long)MIRORR_LTS_NOALLOC_MAX_POINTS) {
    set_error("%lld point pairs exceed the no-allocation LTS limit of %d", n,
              (int)MIRORR_LTS_NOALLOC_MAX_POINTS);
    return MIRORR_ERANGE;
  }
  lts_begin(hs);
  if (n <= 0) {
    lts_finish(hs);
    if (inner_iters) *inner_iters = 0;
    return MIRORR_OK;
  }
  int dev = 0;
  MB2_CUDA_TRY(cudaGetDevice(&dev));
  unsigned char *base = nullptr;
  int max_ctas = 0;
  MB2_TRY(na_setup(dev, &base, &max_ctas));
  if (max_ctas > kNaMaxCtas) max_ctas = kNaMaxCtas;
  long long want = (n + 4 * kThreads - 1) / (4 * kThreads);
  int grid = (int)(want < 1 ? 1 : (want > max_ctas ? max_ctas : want));
  long long counts[2] = {n, 0};
  MB2_CUDA_TRY(cudaMemcpyAsync(base + kNaState, &hs, sizeof(LtsState), cudaMemcpyHostToDevice, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(base + kNaCount, counts, sizeof(counts), cudaMemcpyHostToDevice, st));
  MB2_CUDA_TRY(cudaMemsetAsync(base + kNaHist, 0, sizeof(unsigned int) * 3 * kBins, st));
  MB2_CUDA_TRY(cudaMemsetAsync(base + kNaCtl, 0, sizeof(LtsCtl), st));
  LtsArgs a;
  a.state = reinterpret_cast<LtsState *>(base + kNaState);
  a.init = init_dev;
  a.moved = moved_dev;
  a.n_dev = reinterpret_cast<const long long *>(base + kNaCount);
  a.resid = reinterpret_cast<double *>(base + kNaResid);
  a.partial = reinterpret_cast<double *>(base + kNaPartial);
  a.hist = reinterpret_cast<unsigned int *>(base + kNaHist);
  a.cand = reinterpret_cast<unsigned long long *>(base + kNaCand);
  a.ctl = reinterpret_cast<LtsCtl *>(base + kNaCtl);
  a.spin_limit = kDefaultSpinLimit;
  void *args[] = {&a};
  MB2_CUDA_TRY(cudaLaunchCooperativeKernel((void *)lts_kernel, dim3(grid), dim3(kThreads), args, 0, st));
  ++g_launches;
  LtsCtl ctl;
  MB2_CUDA_TRY(cudaMemcpyAsync(&hs, base + kNaState, sizeof(LtsState), cudaMemcpyDeviceToHost, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(&ctl, base + kNaCtl, sizeof(LtsCtl), cudaMemcpyDeviceToHost, st));
  MB2_CUDA_TRY(cudaStreamSynchronize(st));
  if (ctl.err) {
    set_error("LTS grid barrier timed out");
    return MIRORR_ETIMEOUT;
  }
  if (inner_iters) *inner_iters = hs.iter;
  lts_finish(hs);
  return MIRORR_OK;
}

}  // namespace mb2
