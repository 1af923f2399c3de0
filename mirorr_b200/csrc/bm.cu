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
#include <cuda_fp16.h>

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
// Each thread computes PX consecutive x positions of one row: every footprint
// row of PX + BW - 1 floats is loaded once and serves all PX positions.  Per
// position the statistics are the two-pass ones of normalizedCorrelation
// (mean over all voxels, then the masked sum of squares,
// itkBlockMatcher.txx:57-95).  The mean is an FP64 sum (exact for float
// inputs of ordinary range, so a flat footprint's mean is its value); the
// sum of squares is taken in FP32 about the FP32 mean.  They feed the FP32
// search only, where the one decision that must be exact is Syy = 0.  When
// the FP64 mean is a float, a masked voxel differs from it in FP32 exactly
// when it does in FP64; otherwise an FP32 sum of at least 1e-30 implies a
// non-zero FP64 one, and below that the position is recomputed with the FP64
// two-pass sum, zero exactly when every masked voxel equals the mean, as in
// the reference.
constexpr int kBoxPX = 4;

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
  constexpr int PX = kBoxPX, RL = PX + BW - 1;
  const int ngx = (nx + PX - 1) / PX;
  const long long n = (long long)ngx * ny * nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    int gx, yy, z;
    split3(p, ngx, ny, gx, yy, z);
    const int x0 = gx * PX;
    const long long o = ((long long)z * ny + yy) * nx + x0;
    const bool rowok = yy <= ny - BW && z <= nz - BW;
    double sum[PX], mean[PX], ss[PX];
    bool all_in[PX], ok[PX];
#pragma unroll
    for (int j = 0; j < PX; ++j) {
      sum[j] = 0.0;
      ss[j] = 0.0;
      all_in[j] = true;
      ok[j] = rowok && x0 + j <= nx - BW;
    }
    if (rowok && x0 <= nx - BW) {
#pragma unroll
      for (int vz = 0; vz < BW; ++vz)
#pragma unroll
        for (int vy = 0; vy < BW; ++vy) {
          const float *r = y + o + ((long long)vz * ny + vy) * nx;
          float v[RL];
#pragma unroll
          for (int i = 0; i < RL; ++i) v[i] = (x0 + i < nx) ? __ldg(r + i) : 0.f;
#pragma unroll
          for (int vx = 0; vx < BW; ++vx)
#pragma unroll
            for (int j = 0; j < PX; ++j) sum[j] = __dadd_rn(sum[j], (double)v[j + vx]);
        }
      constexpr int B = BW * BW * BW;
#pragma unroll
      for (int j = 0; j < PX; ++j)
        mean[j] = (B & (B - 1)) == 0 ? sum[j] * (1.0 / B) : __ddiv_rn(sum[j], (double)B);
      float mu[PX], s32[PX];
#pragma unroll
      for (int j = 0; j < PX; ++j) { mu[j] = (float)mean[j]; s32[j] = 0.f; }
      // mask columns of the PX + BW - 1 wide footprint rows: in the mask in
      // every row (allb) and in some row (anyb)
      unsigned int allb = ~0u, anyb = 0u;
#pragma unroll
      for (int vz = 0; vz < BW; ++vz)
#pragma unroll
        for (int vy = 0; vy < BW; ++vy) {
          const long long q = o + ((long long)vz * ny + vy) * nx;
          float v[RL];
          bool m[RL];
          unsigned int mb = 0u;
#pragma unroll
          for (int i = 0; i < RL; ++i) {
            const bool in = x0 + i < nx;
            v[i] = in ? __ldg(y + q + i) : 0.f;
            m[i] = in && __ldg(ms + q + i) != 0;
            mb |= (m[i] ? 1u : 0u) << i;
          }
          allb &= mb;
          anyb |= mb;
#pragma unroll
          for (int vx = 0; vx < BW; ++vx)
#pragma unroll
            for (int j = 0; j < PX; ++j) {
              const float d = m[j + vx] ? v[j + vx] - mu[j] : 0.f;
              s32[j] = fmaf(d, d, s32[j]);
            }
        }
      constexpr unsigned int kRow = (1u << BW) - 1u;
      bool any_in[PX];
#pragma unroll
      for (int j = 0; j < PX; ++j) {
        all_in[j] = ((allb >> j) & kRow) == kRow;
        any_in[j] = ((anyb >> j) & kRow) != 0u;
      }
#pragma unroll
      for (int j = 0; j < PX; ++j) {
        ss[j] = (double)s32[j];
        // no masked voxel: zero; with a mean that is a float, v - mean is zero
        // in FP32 exactly when it is in FP64; otherwise a tiny FP32 sum is
        // recomputed in FP64
        if (ok[j] && any_in[j] && s32[j] < 1e-30f && (double)mu[j] != mean[j])
          ss[j] = box_ss64<BW>(y, ms, o + j, nx, ny, mean[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < PX; ++j) {
      if (x0 + j >= nx) break;
      if (!ok[j]) {
        out[o + j] = make_float2(0.f, 0.f);
      } else {
        const float fs = (float)ss[j];
        out[o + j] = make_float2((float)mean[j], all_in[j] ? fs : -fs);
      }
    }
  }
}

mirorr_status launch_box_stats(const BmGeom &g, const float *search, const uint8_t *smask,
                               float2 *stats, cudaStream_t s) {
  long long n = (long long)((g.size[0] + kBoxPX - 1) / kBoxPX) * g.size[1] * g.size[2];
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

template <typename T>
__global__ void block_variance_kernel(const T *__restrict__ img, int nx, int ny, int nbx,
                                      int nby, int nbz, int stx, int sty, int stz, int G, int bw,
                                      double *__restrict__ var, unsigned long long *__restrict__ key) {
  long long nb = (long long)nbx * nby * nbz;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb;
       b += (long long)gridDim.x * blockDim.x) {
    int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((long long)nbx * nby));
    long long o = ((long long)(stz + bz * G) * ny + (sty + by * G)) * nx + (stx + bx * G);
    double cnt = 0.0, sum = 0.0, ssq = 0.0;
    for (int z = 0; z < bw; ++z)
      for (int y = 0; y < bw; ++y)
        for (int x = 0; x < bw; ++x) {
          float v = to_float(img[o + ((long long)z * ny + y) * nx + x]);
          cnt = __dadd_rn(cnt, 1.0);
          sum = __dadd_rn(sum, (double)v);
          float sq = __fmul_rn(v, v);  // float * float in the reference
          ssq = __dadd_rn(ssq, (double)sq);
        }
    double mean = __ddiv_rn(sum, cnt);
    double v = __dsub_rn(__ddiv_rn(ssq, cnt), __dmul_rn(mean, mean));
    var[b] = v;
    key[b] = order_key(v);
  }
}

// Radix select control block (device memory).
struct SelectCtl {
  unsigned long long prefix;
  unsigned long long mask;
  unsigned long long k;      // rank still to find within the prefix bucket
  unsigned long long n;
};

__global__ void select_hist_kernel(const unsigned long long *__restrict__ key, long long n,
                                   const SelectCtl *__restrict__ ctl, int shift,
                                   unsigned int *__restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  unsigned long long prefix = ctl->prefix, mask = ctl->mask;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned long long k = key[i];
    if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 0xFF], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

// The select's initial state (a kernel rather than a host copy, so the
// sequence can be captured into a graph).
__global__ void select_init_kernel(SelectCtl *ctl, unsigned long long k, unsigned long long n,
                                   unsigned int *hist) {
  if (threadIdx.x == 0) *ctl = SelectCtl{0ULL, 0ULL, k, n};
  hist[threadIdx.x] = 0u;
}

__global__ void select_scan_kernel(SelectCtl *ctl, int shift, unsigned int *hist) {
  __shared__ unsigned int h[256];
  int t = threadIdx.x;
  h[t] = hist[t];
  __syncthreads();
  if (t == 0) {
    unsigned long long k = ctl->k, cum = 0;
    int d = 0;
    for (; d < 256; ++d) {
      if (cum + h[d] > k) break;
      cum += h[d];
    }
    if (d == 256) d = 255;  // cannot happen for k < count
    ctl->k = k - cum;
    ctl->prefix |= ((unsigned long long)d) << shift;
    ctl->mask |= 0xFFULL << shift;
  }
  __syncthreads();
  hist[t] = 0;
}

__global__ void select_flags_kernel(const double *__restrict__ var, long long n,
                                    const SelectCtl *__restrict__ ctl,
                                    uint8_t *__restrict__ selected) {
  unsigned long long p = ctl->prefix;
  unsigned long long u = (p & 0x8000000000000000ULL) ? (p & 0x7FFFFFFFFFFFFFFFULL) : ~p;
  double cutoff = __longlong_as_double((long long)u);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    selected[i] = var[i] > cutoff ? 1 : 0;
}

mirorr_status launch_variance_selection(const BmGeom &g, const void *base, double keep,
                                        BmWork &w, const uint8_t **selected_out,
                                        cudaStream_t s, int dtype) {
  *selected_out = nullptr;
  if (!(keep < 1.0)) return MIRORR_OK;
  long long n = g.nblocks;
  MB2_TRY(w.var.ensure(sizeof(double) * n + sizeof(unsigned long long) * n));
  MB2_TRY(w.selected.ensure(n));
  MB2_TRY(w.select_state.ensure(sizeof(SelectCtl)));
  MB2_TRY(w.hist.ensure(256 * sizeof(unsigned int)));
  double *var = w.var.as<double>();
  unsigned long long *key = reinterpret_cast<unsigned long long *>(var + n);
  int threads = 256;
  long long blocks = (n + threads - 1) / threads;
  if (blocks > (long long)sm_count() * 32) blocks = (long long)sm_count() * 32;
  // the reference's FP64 variance (exact k-th value, so the selected blocks
  // are the reference's for any storage type)
  if (dtype == MIRORR_DTYPE_BF16)
    block_variance_kernel<<<(unsigned)blocks, threads, 0, s>>>(
        static_cast<const __nv_bfloat16 *>(base), g.size[0], g.size[1], g.nb[0], g.nb[1], g.nb[2],
        g.st[0], g.st[1], g.st[2], g.ngap, g.bw, var, key);
  else if (dtype == MIRORR_DTYPE_F16)
    block_variance_kernel<<<(unsigned)blocks, threads, 0, s>>>(
        static_cast<const __half *>(base), g.size[0], g.size[1], g.nb[0], g.nb[1], g.nb[2],
        g.st[0], g.st[1], g.st[2], g.ngap, g.bw, var, key);
  else
    block_variance_kernel<<<(unsigned)blocks, threads, 0, s>>>(
        static_cast<const float *>(base), g.size[0], g.size[1], g.nb[0], g.nb[1], g.nb[2],
        g.st[0], g.st[1], g.st[2], g.ngap, g.bw, var, key);
  MB2_LAUNCH_CHECK();
  // cut-off index (unsigned)((1 - keep) * N); index >= N -> the maximum
  unsigned long long idx = (unsigned long long)(unsigned int)((1.0 - keep) * (double)n);
  if (idx >= (unsigned long long)n) idx = n - 1;
  SelectCtl *ctl = w.select_state.as<SelectCtl>();
  select_init_kernel<<<1, 256, 0, s>>>(ctl, idx, (unsigned long long)n, w.hist.as<unsigned int>());
  MB2_LAUNCH_CHECK();
  for (int pass = 0; pass < 8; ++pass) {
    int shift = 56 - 8 * pass;
    select_hist_kernel<<<(unsigned)blocks, threads, 0, s>>>(key, n, ctl, shift,
                                                            w.hist.as<unsigned int>());
    MB2_LAUNCH_CHECK();
    select_scan_kernel<<<1, 256, 0, s>>>(ctl, shift, w.hist.as<unsigned int>());
    MB2_LAUNCH_CHECK();
  }
  select_flags_kernel<<<(unsigned)blocks, threads, 0, s>>>(var, n, ctl, w.selected.as<uint8_t>());
  MB2_LAUNCH_CHECK();
  *selected_out = w.selected.as<uint8_t>();
  return MIRORR_OK;
}

// ---------------------------------------------------------------------------
// 4. post-filter + compaction
// ---------------------------------------------------------------------------
constexpr int kTile = 2048;  // blocks per compaction tile (256 threads x 8)

__device__ inline bool keep_block(const BmOut &o, long long b) {
  if (!(o.status[b] & 1)) return false;
  double cb = (double)o.best[b], c2 = (double)o.second[b];
  return cb > 1e-7 && fabs(cb - c2) > 1e-4;
}

__device__ void pf_count_tile(const BmOut &o, long long n, unsigned int *tile_count, long long tile) {
  __shared__ unsigned int cnt;
  __syncthreads();
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  long long t0 = tile * kTile;
  unsigned int c = 0;
  for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
    long long b = t0 + i;
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
