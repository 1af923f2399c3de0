// bm.cu -- block-matching kernels for sm_100a (plain FP32 path).
//
// One matcher call (AbstractBlockMatcher::GetOffsets) runs:
//   1. box_stats:   per candidate origin p of the search image, the block mean
//                   mu(p) (over all BW^3 voxels, unmasked, as
//                   itkBlockMatcher.txx:57-68) and the masked sum of squares
//                   Syy(p) = sum_{ms != 0} (y - mu)^2, both in FP64 in the
//                   reference's raster order, stored as float2; the sign bit
//                   of Syy is set when a search-mask voxel of the footprint is 0.
//   2. selection:   (optional) dead-code variance cut-off of
//                   itkBlockMatcher.txx:664-719, FP64 per block, exact k-th
//                   value by a device radix select.
//   3. ncc:         the search itself (ncc.cu).
//   4. postfilter:  best > 1e-7 && |best - second| > 1e-4 (itkBlockMatcher.txx:884-918),
//                   deterministic raster-order compaction and block -> mm points
//                   (itkAbstractBlockMatcher.h:271-287).
#include <cuda_bf16.h>
#include <type_traits>
#include <cuda_fp16.h>

#include "gridsel.cuh"
#include "kernels.cuh"

namespace mb2 {

bool bm_geometry(const int size[3], int bw, int bgap, int ngap, int nw, BmGeom &g) {
  if (bw <= 0 || bgap <= 0 || ngap <= 0 || nw <= 0) return false;
  g.nblocks = 1;
  for (int d = 0; d < 3; ++d) {
    if (size[d] < bw) return false;
    g.size[d] = size[d];
    int n = (size[d] - bw) / ngap + 1;
    int region = ngap * (n - 1) + bw;
    g.nb[d] = n;
    g.st[d] = (size[d] - region) / 2;
    g.nblocks *= n;
  }
  g.bw = bw;
  g.bgap = bgap;
  g.ngap = ngap;
  g.nw = nw;
  return true;
}

void point_geom(const double origin[3], const double spacing[3], const double direction[9],
                int bw, PointGeom &pg) {
  for (int r = 0; r < 3; ++r) {
    pg.origin[r] = origin[r];
    for (int c = 0; c < 3; ++c) pg.a[3 * r + c] = direction[3 * r + c] * spacing[c];
    pg.half[r] = spacing[r] * (0.5 * (double)bw);
  }
}

// ---------------------------------------------------------------------------
// 1. box statistics
// ---------------------------------------------------------------------------
// Each thread computes PZ consecutive z positions of one (x, y) column, and
// the lanes of a warp take consecutive x: every footprint row load is a
// coalesced warp-wide read, and each of the PZ + BW - 1 window planes' rows is
// loaded once for all PZ positions.  Per position the statistics are the
// two-pass ones of normalizedCorrelation (mean over all voxels, then the
// masked sum of squares, itkBlockMatcher.txx:57-95), both accumulated in the
// reference's raster order (vz, vy, vx) whatever the interleaving across
// positions.  The mean is an FP64 sum (exact for float inputs of ordinary
// range, so a flat footprint's mean is its value); the sum of squares is
// taken in FP32 about the FP32 mean.  They feed the FP32 search only, where
// the one decision that must be exact is Syy = 0.  When the FP64 mean is a
// float, a masked voxel differs from it in FP32 exactly when it does in FP64;
// otherwise an FP32 sum of at least 1e-30 implies a non-zero FP64 one, and
// below that the position is recomputed with the FP64 two-pass sum, zero
// exactly when every masked voxel equals the mean, as in the reference.
constexpr int kBoxPZ = 8;

// FP64 masked sum of squares about mean of the footprint at linear index o
// (raster order, fused multiply-adds); the footprint lies inside the volume.
template <int BW>
__device__ __noinline__ double box_ss64(const float *__restrict__ y,
                                        const uint8_t *__restrict__ ms, long long o, int nx,
                                        int ny, double mean) {
  double ss = 0.0;
  for (int vz = 0; vz < BW; ++vz)
    for (int vy = 0; vy < BW; ++vy) {
      const long long q = o + ((long long)vz * ny + vy) * nx;
      for (int vx = 0; vx < BW; ++vx)
        if (__ldg(ms + q + vx)) {
          const double d = __dsub_rn((double)__ldg(y + q + vx), mean);
          ss = __fma_rn(d, d, ss);
        }
    }
  return ss;
}

template <int BW>
__global__ void __launch_bounds__(256) box_stats_kernel(const float *__restrict__ y,
                                                        const uint8_t *__restrict__ ms, int nx,
                                                        int ny, int nz, float2 *__restrict__ out) {
  constexpr int PZ = kBoxPZ, NP = PZ + BW - 1;
  const int ngz = (nz + PZ - 1) / PZ;
  const long long n = (long long)nx * ny * ngz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    int x, yy, gz;
    split3(p, nx, ny, x, yy, gz);
    const int z0 = gz * PZ;
    const long long o = ((long long)z0 * ny + yy) * nx + x;
    const long long plane = (long long)nx * ny;
    const bool colok = x <= nx - BW && yy <= ny - BW;
    // planes z0 .. zend - 1 are read; positions z0 + j <= nz - BW are valid
    const int zend = min(z0 + NP, nz);
    double sum[PZ], mean[PZ];
    float s32[PZ];
    bool all_in[PZ], any_in[PZ], ok[PZ];
#pragma unroll
    for (int j = 0; j < PZ; ++j) {
      sum[j] = 0.0;
      s32[j] = 0.f;
      all_in[j] = true;
      any_in[j] = false;
      ok[j] = colok && z0 + j <= nz - BW;
    }
    if (ok[0]) {
#pragma unroll
      for (int wz = 0; wz < NP; ++wz) {
        if (z0 + wz >= zend) break;
#pragma unroll
        for (int vy = 0; vy < BW; ++vy) {
          const float *r = y + o + wz * plane + (long long)vy * nx;
          float v[BW];
#pragma unroll
          for (int vx = 0; vx < BW; ++vx) v[vx] = __ldg(r + vx);
#pragma unroll
          for (int j = 0; j < PZ; ++j) {
            const int vz = wz - j;
            if (vz < 0 || vz >= BW) continue;
#pragma unroll
            for (int vx = 0; vx < BW; ++vx) sum[j] = __dadd_rn(sum[j], (double)v[vx]);
          }
        }
      }
      constexpr int B = BW * BW * BW;
      float mu[PZ];
#pragma unroll
      for (int j = 0; j < PZ; ++j) {
        mean[j] = (B & (B - 1)) == 0 ? sum[j] * (1.0 / B) : __ddiv_rn(sum[j], (double)B);
        mu[j] = (float)mean[j];
      }
#pragma unroll
      for (int wz = 0; wz < NP; ++wz) {
        if (z0 + wz >= zend) break;
#pragma unroll
        for (int vy = 0; vy < BW; ++vy) {
          const long long q = o + wz * plane + (long long)vy * nx;
          float v[BW];
          bool m[BW];
          bool rall = true, rany = false;
#pragma unroll
          for (int vx = 0; vx < BW; ++vx) {
            v[vx] = __ldg(y + q + vx);
            m[vx] = __ldg(ms + q + vx) != 0;
            rall = rall && m[vx];
            rany = rany || m[vx];
          }
#pragma unroll
          for (int j = 0; j < PZ; ++j) {
            const int vz = wz - j;
            if (vz < 0 || vz >= BW) continue;
            all_in[j] = all_in[j] && rall;
            any_in[j] = any_in[j] || rany;
#pragma unroll
            for (int vx = 0; vx < BW; ++vx) {
              const float d = m[vx] ? v[vx] - mu[j] : 0.f;
              s32[j] = fmaf(d, d, s32[j]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < PZ; ++j) {
      if (z0 + j >= nz) break;
      float2 r = make_float2(0.f, 0.f);
      if (ok[j]) {
        double ss = (double)s32[j];
        // no masked voxel: zero; with a mean that is a float, v - mean is zero
        // in FP32 exactly when it is in FP64; otherwise a tiny FP32 sum is
        // recomputed in FP64
        if (any_in[j] && s32[j] < 1e-30f && (double)(float)mean[j] != mean[j])
          ss = box_ss64<BW>(y, ms, o + j * plane, nx, ny, mean[j]);
        const float fs = (float)ss;
        r = make_float2((float)mean[j], all_in[j] ? fs : -fs);
      }
      out[o + j * plane] = r;
    }
  }
}

mirorr_status launch_box_stats(const BmGeom &g, const float *search, const uint8_t *smask,
                               float2 *stats, cudaStream_t s) {
  long long n = (long long)g.size[0] * g.size[1] * ((g.size[2] + kBoxPZ - 1) / kBoxPZ);
  int threads = 256;
  long long blocks = (n + threads - 1) / threads;
  if (blocks > (long long)sm_count() * 64) blocks = (long long)sm_count() * 64;
  switch (g.bw) {
#define CASE(B) \
  case B: box_stats_kernel<B><<<(unsigned)blocks, threads, 0, s>>>(search, smask, g.size[0], g.size[1], g.size[2], stats); break;
    CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
#undef CASE
    default:
      set_error("block width %d not supported (1..8)", g.bw);
      return MIRORR_EINVAL;
  }
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

// ---------------------------------------------------------------------------
// 2. variance selection
// ---------------------------------------------------------------------------
__device__ inline unsigned long long order_key(double v) {
  unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
}

__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_float(__half v) { return __half2float(v); }

// The whole selection in one cooperative launch (CTAs meet at a grid barrier
// whose wait is bounded):
//   1. per block (one thread each) the variance as the reference computes it
//      (itkBlockMatcher.txx:664-719: FP64 count, sum and sum of float
//      squares in raster order, var = ssq / cnt - mean^2), its order key, and
//      a histogram of the keys' top 12 bits;
//   2. an MSD radix select of the key of rank idx: while more than one CTA's
//      worth of keys share the prefix, the next 12 bits are histogrammed;
//      then those keys are gathered and ranked by counting;
//   3. selected[b] = var[b] > the selected value.
constexpr int kSelThreads = 256;
constexpr int kSelBins = 4096;
constexpr int kSelCand = kSelThreads;

// Device control block of one selection, followed in memory by 3 * kSelBins
// histogram words; the launcher zeroes both.
struct SelectCtl {
  unsigned int bar_count;
  unsigned int bar_gen;
  int err;
  int pad;
  unsigned long long ncand;
};

struct SelectArgs {
  const void *img;
  int nx, ny, nbx, nby, nbz, stx, sty, stz, G, bw;
  long long n;
  unsigned long long idx;  // rank of the cut-off value (ascending)
  double *var;
  unsigned long long *key;
  unsigned long long *cand;  // kSelCand
  SelectCtl *ctl;
  unsigned int *hist;        // 3 * kSelBins
  uint8_t *selected;
  unsigned int *give_up;     // set when a barrier wait gives up (may be null)
  long long spin_limit;
};

// BW > 0: the block width known at compile time (the 64 or 125 loads of a
// block are all issued before the sums); BW = 0: a.bw at run time.
template <typename T, int BW>
__device__ inline double block_variance(const T *__restrict__ img, const SelectArgs &a,
                                        long long b) {
  const int bw = BW > 0 ? BW : a.bw;
  const int bx = (int)(b % a.nbx), by = (int)((b / a.nbx) % a.nby);
  const int bz = (int)(b / ((long long)a.nbx * a.nby));
  const long long o =
      ((long long)(a.stz + bz * a.G) * a.ny + (a.sty + by * a.G)) * a.nx + (a.stx + bx * a.G);
  double cnt = 0.0, sum = 0.0, ssq = 0.0;
#pragma unroll
  for (int z = 0; z < bw; ++z)
#pragma unroll
    for (int y = 0; y < bw; ++y)
#pragma unroll
      for (int x = 0; x < bw; ++x) {
        const float v = to_float(img[o + ((long long)z * a.ny + y) * a.nx + x]);
        cnt = __dadd_rn(cnt, 1.0);
        sum = __dadd_rn(sum, (double)v);
        const float sq = __fmul_rn(v, v);  // float * float in the reference
        ssq = __dadd_rn(ssq, (double)sq);
      }
  const double mean = __ddiv_rn(sum, cnt);
  return __dsub_rn(__ddiv_rn(ssq, cnt), __dmul_rn(mean, mean));
}

template <typename T>
__global__ void __launch_bounds__(kSelThreads) select_kernel(SelectArgs a) {
  __shared__ unsigned int h[kSelBins];
  __shared__ unsigned long long ck[kSelCand];
  __shared__ unsigned long long s_pair[2];
  __shared__ unsigned long long s_cut;
  __shared__ unsigned long long s_nc;
  const T *img = static_cast<const T *>(a.img);
  const long long n = a.n;
  const long long gstride = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned int nctas = gridDim.x;
  SelectCtl *ctl = a.ctl;
  // ---- 1. variances, keys, histogram of the top 12 bits --------------------
  for (int i = threadIdx.x; i < kSelBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (long long b = gtid; b < n; b += gstride) {
    const double v = a.bw == 4   ? block_variance<T, 4>(img, a, b)
                     : a.bw == 5 ? block_variance<T, 5>(img, a, b)
                                 : block_variance<T, 0>(img, a, b);
    const unsigned long long k = order_key(v);
    a.var[b] = v;
    a.key[b] = k;
    hist_add(h, (unsigned)(k >> 52));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kSelBins; i += blockDim.x)
    if (h[i]) atomicAdd(&a.hist[i], h[i]);
  bool ok = grid_barrier(&ctl->bar_count, &ctl->bar_gen, &ctl->err, a.spin_limit, nctas);
  // ---- 2. radix select of rank idx -----------------------------------------
  unsigned long long k = a.idx, prefix = 0, mask = 0;
  int shift = 52, bits = 12, pass = 0;
  while (ok) {
    // every CTA scans the global histogram of this pass identically
    const unsigned int *gh = a.hist + (pass % 3) * kSelBins;
    for (int i = threadIdx.x; i < kSelBins; i += blockDim.x) h[i] = __ldcg(&gh[i]);
    __syncthreads();
    int d = 0;
    unsigned long long cum = 0;
    find_bucket<kSelBins, kSelThreads>(h, k, 1 << bits, s_pair, &d, &cum);
    const unsigned long long bucket = h[d];
    k -= cum;
    prefix |= (unsigned long long)d << shift;
    mask |= ((1ULL << bits) - 1ULL) << shift;
    __syncthreads();
    if (bucket <= (unsigned long long)kSelCand || shift == 0) break;
    // more than one CTA's worth of keys share the prefix: the next bits
    ++pass;
    bits = shift >= 12 ? 12 : shift;
    shift -= bits;
    if (blockIdx.x == 0) {
      unsigned int *zb = a.hist + ((pass + 1) % 3) * kSelBins;
      for (int i = threadIdx.x; i < kSelBins; i += blockDim.x) zb[i] = 0;
    }
    for (int i = threadIdx.x; i < kSelBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (long long i = gtid; i < n; i += gstride) {
      const unsigned long long key = a.key[i];
      if ((key & mask) == prefix) hist_add(h, (unsigned)(key >> shift) & ((1u << bits) - 1u));
    }
    __syncthreads();
    unsigned int *gh2 = a.hist + (pass % 3) * kSelBins;
    for (int i = threadIdx.x; i < kSelBins; i += blockDim.x)
      if (h[i]) atomicAdd(&gh2[i], h[i]);
    ok = grid_barrier(&ctl->bar_count, &ctl->bar_gen, &ctl->err, a.spin_limit, nctas);
  }
  if (ok && shift != 0) {
    // the bucket's keys (at most one per thread of a CTA), ranked by counting
    for (long long i = gtid; i < n; i += gstride) {
      const unsigned long long key = a.key[i];
      if ((key & mask) == prefix) {
        const unsigned long long pos = atomicAdd(&ctl->ncand, 1ULL);
        if (pos < (unsigned long long)kSelCand) a.cand[pos] = key;
      }
    }
    ok = grid_barrier(&ctl->bar_count, &ctl->bar_gen, &ctl->err, a.spin_limit, nctas);
    if (ok) {
      if (threadIdx.x == 0) {
        s_nc = __ldcg(&ctl->ncand);
        s_cut = prefix;
      }
      __syncthreads();
      const int nc = (int)(s_nc < (unsigned long long)kSelCand ? s_nc : kSelCand);
      const unsigned long long kk = k < (unsigned long long)nc ? k : (nc > 0 ? nc - 1 : 0);
      for (int i = threadIdx.x; i < nc; i += blockDim.x) ck[i] = __ldcg(&a.cand[i]);
      __syncthreads();
      if (threadIdx.x < nc) {
        const unsigned long long v = ck[threadIdx.x];
        int lo = 0, eq = 0;
        for (int j = 0; j < nc; ++j) {
          lo += ck[j] < v;
          eq += ck[j] == v;
        }
        if ((unsigned long long)lo <= kk && kk < (unsigned long long)(lo + eq)) s_cut = v;
      }
      __syncthreads();
      prefix = s_cut;
    }
  }
  if (!ok) {
    if (threadIdx.x == 0 && a.give_up) atomicExch(a.give_up, 1u);
    return;
  }
  // ---- 3. flags --------------------------------------------------------------
  const unsigned long long u =
      (prefix & 0x8000000000000000ULL) ? (prefix & 0x7FFFFFFFFFFFFFFFULL) : ~prefix;
  const double cutoff = __longlong_as_double((long long)u);
  for (long long b = gtid; b < n; b += gstride) a.selected[b] = a.var[b] > cutoff ? 1 : 0;
}

template <typename T>
mirorr_status launch_select(SelectArgs &a, cudaStream_t s) {
  static int per_sm[3] = {0, 0, 0};
  const int slot = std::is_same<T, float>::value ? 0 : (std::is_same<T, __half>::value ? 2 : 1);
  if (per_sm[slot] == 0) {
    int per = 0;
    MB2_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, select_kernel<T>, kSelThreads, 0));
    per_sm[slot] = per > 0 ? per : 1;
  }
  long long want = (a.n + 4 * kSelThreads - 1) / (4 * kSelThreads);
  const long long cap = (long long)sm_count() * per_sm[slot];
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  void *args[] = {&a};
  MB2_CUDA_TRY(cudaLaunchCooperativeKernel((void *)select_kernel<T>, dim3((unsigned)want),
                                           dim3(kSelThreads), args, 0, s));
  ++g_launches;
  return MIRORR_OK;
}

size_t selection_var_bytes(long long nblocks) {
  return sizeof(double) * nblocks + sizeof(unsigned long long) * (nblocks + kSelCand);
}

size_t selection_state_bytes() { return sizeof(SelectCtl) + sizeof(unsigned int) * 3 * kSelBins; }

mirorr_status launch_variance_selection(const BmGeom &g, const void *base, double keep,
                                        BmWork &w, const uint8_t **selected_out,
                                        cudaStream_t s, int dtype, unsigned int *give_up,
                                        long long spin_limit) {
  *selected_out = nullptr;
  if (!(keep < 1.0)) return MIRORR_OK;
  long long n = g.nblocks;
  MB2_TRY(w.var.ensure(selection_var_bytes(n)));
  MB2_TRY(w.selected.ensure(n));
  const size_t ctl_bytes = selection_state_bytes();
  MB2_TRY(w.select_state.ensure(ctl_bytes));
  SelectArgs a;
  a.img = base;
  a.nx = g.size[0]; a.ny = g.size[1];
  a.nbx = g.nb[0]; a.nby = g.nb[1]; a.nbz = g.nb[2];
  a.stx = g.st[0]; a.sty = g.st[1]; a.stz = g.st[2];
  a.G = g.ngap; a.bw = g.bw;
  a.n = n;
  // cut-off index (unsigned)((1 - keep) * N); index >= N -> the maximum
  unsigned long long idx = (unsigned long long)(unsigned int)((1.0 - keep) * (double)n);
  if (idx >= (unsigned long long)n) idx = n - 1;
  a.idx = idx;
  a.var = w.var.as<double>();
  a.key = reinterpret_cast<unsigned long long *>(a.var + n);
  a.cand = a.key + n;
  a.ctl = w.select_state.as<SelectCtl>();
  a.hist = reinterpret_cast<unsigned int *>(a.ctl + 1);
  a.selected = w.selected.as<uint8_t>();
  a.give_up = give_up;
  a.spin_limit = spin_limit > 0 ? spin_limit : 1LL << 23;  // default: about 0.84 s of polling
  // a memset, not a host copy, so the sequence can be captured into a graph
  MB2_CUDA_TRY(cudaMemsetAsync(w.select_state.ptr, 0, ctl_bytes, s));
  // the reference's FP64 variance (exact k-th value, so the selected blocks
  // are the reference's for any storage type)
  if (dtype == MIRORR_DTYPE_BF16) MB2_TRY(launch_select<__nv_bfloat16>(a, s));
  else if (dtype == MIRORR_DTYPE_F16) MB2_TRY(launch_select<__half>(a, s));
  else MB2_TRY(launch_select<float>(a, s));
  *selected_out = w.selected.as<uint8_t>();
  return MIRORR_OK;
}

// ---------------------------------------------------------------------------
// 4. post-filter + compaction
// ---------------------------------------------------------------------------
constexpr int kTile = 2048;  // blocks per compaction tile (256 threads x 8)

// The three reads are unconditional (every block has a status and scores),
// so a thread's blocks are all read before the tests.
__device__ inline bool keep_block(const BmOut &o, long long b) {
  const uint8_t st = o.status[b];
  const double cb = (double)o.best[b], c2 = (double)o.second[b];
  return (st & 1) && cb > 1e-7 && fabs(cb - c2) > 1e-4;
}

__device__ void pf_count_tile(const BmOut &o, long long n, unsigned int *tile_count, long long tile) {
  __shared__ unsigned int cnt;
  __syncthreads();
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  long long t0 = tile * kTile;
  unsigned int c = 0;
#pragma unroll
  for (int k = 0; k < kTile / 256; ++k) {  // 256 threads per CTA
    long long b = t0 + threadIdx.x + 256 * k;
    if (b < n && keep_block(o, b)) ++c;
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) tile_count[tile] = cnt;
}

__global__ void pf_count_kernel(BmOut o, long long n, unsigned int *tile_count) {
  pf_count_tile(o, n, tile_count, blockIdx.x);
}

__device__ void pf_scan_body(unsigned int *tile_count, long long ntiles, long long *total) {
  // single CTA, 1024 threads: exclusive scan in place (tile counts -> offsets)
  __shared__ unsigned long long carry;
  __shared__ unsigned long long warp_sums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long base = 0; base < ntiles; base += blockDim.x) {
    long long i = base + threadIdx.x;
    unsigned long long v = (i < ntiles) ? tile_count[i] : 0;
    unsigned long long x = v;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      unsigned long long w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, w, off);
        if (lane >= off) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    unsigned long long excl = x - v + (wid > 0 ? warp_sums[wid - 1] : 0) + carry;
    if (i < ntiles) tile_count[i] = (unsigned int)excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = (long long)carry;
}

__global__ void pf_scan_kernel(unsigned int *tile_count, long long ntiles, long long *total) {
  pf_scan_body(tile_count, ntiles, total);
}

__device__ inline void block_point(const PointGeom &pg, int ix, int iy, int iz, double *out) {
  const double idx[3] = {(double)ix, (double)iy, (double)iz};
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    double v = pg.origin[r];
#pragma unroll
    for (int c = 0; c < 3; ++c) v = __dadd_rn(v, __dmul_rn(pg.a[3 * r + c], idx[c]));
    out[r] = __dadd_rn(v, pg.half[r]);
  }
}

__device__ void pf_write_tile(const BmOut &o, long long n, const unsigned int *tile_off,
                              const BmGeom &g, const PointGeom &pg, double *pts_base,
                              double *pts_match, const long long *offset_dev, long long tile) {
  __shared__ unsigned int wsum[8];
  __syncthreads();
  const int per = kTile / 256;  // 8 consecutive blocks per thread
  long long t0 = tile * kTile + (long long)threadIdx.x * per;
  unsigned int flags = 0, c = 0;
#pragma unroll
  for (int k = 0; k < per; ++k) {
    long long b = t0 + k;
    if (b < n && keep_block(o, b)) {
      flags |= 1u << k;
      ++c;
      o.status[b] |= 2;
    }
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned int x = c;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    unsigned int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  unsigned int before = 0;
  for (int w = 0; w < wid; ++w) before += wsum[w];
  unsigned long long pos = (unsigned long long)tile_off[tile] + before + x - c;
  if (!pts_base) return;
  if (offset_dev) pos += (unsigned long long)*offset_dev;
  for (int k = 0; k < per; ++k) {
    if (!(flags & (1u << k))) continue;
    long long b = t0 + k;
    int bx = (int)(b % g.nb[0]), by = (int)((b / g.nb[0]) % g.nb[1]),
        bz = (int)(b / ((long long)g.nb[0] * g.nb[1]));
    int ox = g.st[0] + bx * g.ngap, oy = g.st[1] + by * g.ngap, oz = g.st[2] + bz * g.ngap;
    int m = o.match[b];
    int mx = m % g.size[0], my = (m / g.size[0]) % g.size[1], mz = m / (g.size[0] * g.size[1]);
    block_point(pg, ox, oy, oz, pts_base + 3 * pos);
    block_point(pg, mx, my, mz, pts_match + 3 * pos);
    ++pos;
  }
}

__global__ void pf_write_kernel(BmOut o, long long n, const unsigned int *tile_off, BmGeom g,
                                PointGeom pg, double *pts_base, double *pts_match,
                                const long long *offset_dev) {
  pf_write_tile(o, n, tile_off, g, pg, pts_base, pts_match, offset_dev, blockIdx.x);
}

// ---- the post-filter of many matcher calls in three launches (grid.y = call)
__global__ void pf_count_batch_kernel(const PfCall *calls) {
  const PfCall &c = calls[blockIdx.y];
  if (!c.active) return;
  const long long nt = (c.g.nblocks + kTile - 1) / kTile;
  for (long long t = blockIdx.x; t < nt; t += gridDim.x) pf_count_tile(c.out, c.g.nblocks, c.tiles, t);
}
__global__ void pf_scan_batch_kernel(const PfCall *calls) {
  const PfCall &c = calls[blockIdx.y];
  if (!c.active) return;
  pf_scan_body(c.tiles, (c.g.nblocks + kTile - 1) / kTile, c.count);
}
__global__ void pf_write_batch_kernel(const PfCall *calls) {
  const PfCall &c = calls[blockIdx.y];
  if (!c.active) return;
  const long long nt = (c.g.nblocks + kTile - 1) / kTile;
  for (long long t = blockIdx.x; t < nt; t += gridDim.x)
    pf_write_tile(c.out, c.g.nblocks, c.tiles, c.g, c.pg, c.pts_b, c.pts_m, c.offset, t);
}

mirorr_status launch_postfilter_batch(const PfCall *dev_calls, int ncalls, long long max_blocks,
                                      cudaStream_t s) {
  if (ncalls <= 0) return MIRORR_OK;
  long long nt = (max_blocks + kTile - 1) / kTile;
  if (nt < 1) nt = 1;
  const long long cap = (long long)sm_count() * 4;
  const unsigned gx = (unsigned)(nt < cap ? nt : cap);
  pf_count_batch_kernel<<<dim3(gx, ncalls), 256, 0, s>>>(dev_calls);
  MB2_LAUNCH_CHECK();
  pf_scan_batch_kernel<<<dim3(1, ncalls), 1024, 0, s>>>(dev_calls);
  MB2_LAUNCH_CHECK();
  pf_write_batch_kernel<<<dim3(gx, ncalls), 256, 0, s>>>(dev_calls);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

mirorr_status launch_postfilter(const BmGeom &g, const BmOut &out, BmWork &w,
                                const PointGeom &pg, double *pts_base, double *pts_match,
                                long long *count_dev, const long long *offset_dev,
                                cudaStream_t s) {
  long long n = g.nblocks;
  long long ntiles = (n + kTile - 1) / kTile;
  MB2_TRY(w.tiles.ensure(sizeof(unsigned int) * (ntiles + 1)));
  unsigned int *tiles = w.tiles.as<unsigned int>();
  pf_count_kernel<<<(unsigned)ntiles, 256, 0, s>>>(out, n, tiles);
  MB2_LAUNCH_CHECK();
  pf_scan_kernel<<<1, 1024, 0, s>>>(tiles, ntiles, count_dev);
  MB2_LAUNCH_CHECK();
  pf_write_kernel<<<(unsigned)ntiles, 256, 0, s>>>(out, n, tiles, g, pg, pts_base, pts_match,
                                                    offset_dev);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace mb2
