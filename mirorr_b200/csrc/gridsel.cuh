// gridsel.cuh -- grid-wide primitives shared by the cooperative kernels (the
// LTS fit and the block variance selection): a software grid barrier whose
// wait is bounded, a warp-aggregated add into a shared histogram, and the
// search of a shared histogram for the bucket holding rank k.
#pragma once

#include <cuda_runtime.h>

namespace mb2 {

// Grid barrier over `nctas` co-resident CTAs on (count, gen, err) in global
// memory.  A wait that exceeds `spin_limit` polls (100 ns back-off after the
// first 256) raises *err; every CTA then leaves its barriers at once.  Returns
// false once *err is set.
__device__ inline bool grid_barrier(unsigned int *count, unsigned int *gen_ptr, int *err,
                                    long long spin_limit, unsigned int nctas) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *genp = gen_ptr;
    volatile int *errp = err;
    unsigned int gen = *genp;
    __threadfence();
    unsigned int arrived = atomicAdd(count, 1u) + 1u;
    if (arrived == nctas) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen_ptr, 1u);
    } else {
      long long spins = 0;
      while (*genp == gen && *errp == 0) {
        if (spins > 256) __nanosleep(100);
        if (++spins > spin_limit) {
          atomicExch(err, 1);
          break;
        }
      }
    }
    __threadfence();
    s_ok = (*errp == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

// Adds 1 to bin of a shared histogram, one atomic per group of lanes of the
// warp that hit the same bin.
__device__ inline void hist_add(unsigned int *h, unsigned int bin) {
  const unsigned active = __activemask();
  const unsigned same = __match_any_sync(active, bin);
  if ((threadIdx.x & 31) == (unsigned)(__ffs(same) - 1)) atomicAdd(&h[bin], (unsigned)__popc(same));
}

// Bucket of rank k in the shared histogram h[0, NBINS) of a CTA of NTHREADS:
// the bin d with cum(d) <= k < cum(d) + h[d] (cum = sum of the bins below d),
// found with a block-wide scan.  Returns d in *d_out and cum(d) in *cum_out
// (every thread); k beyond the count gives the last bin nb - 1 and the total.
template <int NBINS, int NTHREADS>
__device__ inline void find_bucket(const unsigned int *h, unsigned long long k, int nb,
                                   unsigned long long *s_pair, int *d_out,
                                   unsigned long long *cum_out) {
  constexpr int kPer = NBINS / NTHREADS;  // bins per thread
  __shared__ unsigned long long s_wsum[NTHREADS / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  unsigned long long local = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) local += h[t * kPer + i];
  unsigned long long inc = local;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    unsigned long long o = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += o;
  }
  if (lane == 31) s_wsum[wid] = inc;
  if (t == 0) { s_pair[0] = ~0ULL; s_pair[1] = 0; }
  __syncthreads();
  unsigned long long wbase = 0;
  for (int w = 0; w < wid; ++w) wbase += s_wsum[w];
  const unsigned long long base = wbase + inc - local;
  if (local > 0 && base <= k && k < base + local) {
    unsigned long long cum = base;
    int d = t * kPer;
    for (int i = 0; i < kPer; ++i, ++d) {
      if (cum + h[d] > k) break;
      cum += h[d];
    }
    s_pair[0] = (unsigned long long)d;
    s_pair[1] = cum;
  }
  __syncthreads();
  if (s_pair[0] == ~0ULL) {
    unsigned long long total = 0;
    for (int w = 0; w < NTHREADS / 32; ++w) total += s_wsum[w];
    *d_out = nb - 1;
    *cum_out = total;
  } else {
    *d_out = (int)s_pair[0];
    *cum_out = s_pair[1];
  }
  __syncthreads();
}

}  // namespace mb2
