// ncc.cu -- exhaustive per-block NCC search for sm_100a.
//
// Semantics (itkBlockMatcher.txx:631-848, normalizedCorrelation :46-101):
// for each block of the grid, every candidate origin p of its clipped +-R
// window (raster order, x fastest) is scored with the squared NCC
//     mu_x, mu_y : means over all BW^3 voxels (unmasked),
//     m          : base mask != 0 && search mask != 0,
//     Sxy = sum m (x - mu_x)(y - mu_y),  Sxx = sum m (x - mu_x)^2,  Syy = sum m (y - mu_y)^2,
//     score = Sxy^2 / Sxx / Syy, or -2 when Sxx <= 0 or Syy <= 0,
// and a running best / second-best is kept in float storage
//     if (best < s) { second = best; best = s; arg = p } else if (second < s) second = s
// starting from -3.
//
// Implementation: a two-stage search.
//   1. FP32 scores of all candidates (the throughput stage).  The window
//      mean and masked sum of squares of each candidate come from box_stats.
//   2. Exact refinement.  Every candidate whose FP32 score lies within 2*delta
//      of the FP32 second-best (delta bounds the FP32 error) is re-scored in
//      FP64 with the reference's arithmetic and summation order, and the
//      reference's sequential best/second update is replayed over them in
//      raster order.  No other candidate can be the best or the second-best,
//      so best, second and argmax equal those of the FP64 reference.
//   Blocks whose candidate list overflows go to a fallback kernel that
//   re-scores their whole window in FP64.
#include "kernels.cuh"

namespace mb2 {

namespace {

constexpr int kLMax = 64;          // refinement list per block
constexpr float kDelta = 1e-4f;    // bound on |FP32 score - FP64 score|

struct NccArgs {
  const float *base;
  const uint8_t *bmask;
  const float *search;
  const uint8_t *smask;
  const float2 *stats;
  const uint8_t *selected;
  int nx, ny, nz;
  int nbx, nby, nbz;
  int stx, sty, stz;
  int G, g, W;
  int emax;
  long long nblocks;
  float *best;
  float *second;
  int32_t *match;
  uint8_t *status;
  unsigned long long *ncc_count;
  int *ovf_list;
  unsigned int *ctl;  // [0] overflow count, [1] refined candidates, [2] fallback blocks
};

__device__ inline void window_axis(int o, int S, int W, int g, int bw, int &s, int &n) {
  int st = o - (W / 2) * g;
  int en = st + W * g;
  int lim = S - bw + 1;
  if (st < 0) st += ((-st + g - 1) / g) * g;
  if (en > lim) en -= ((en - lim + g - 1) / g) * g;
  s = st;
  n = (en > st) ? (en - st + g - 1) / g : 0;
}

// Geometry of one block's search, shared by the kernels.
struct BlockWin {
  long long b;
  int ox, oy, oz;
  int sx, sy, sz;
  int nx, ny, nz;   // candidates per axis
  int ex, ey, ez;   // staged window extent
  int nc;
};

__device__ inline bool block_window(const NccArgs &a, long long b, int bw, BlockWin &w) {
  w.b = b;
  int bx = (int)(b % a.nbx), by = (int)((b / a.nbx) % a.nby), bz = (int)(b / ((long long)a.nbx * a.nby));
  w.ox = a.stx + bx * a.G;
  w.oy = a.sty + by * a.G;
  w.oz = a.stz + bz * a.G;
  window_axis(w.ox, a.nx, a.W, a.g, bw, w.sx, w.nx);
  window_axis(w.oy, a.ny, a.W, a.g, bw, w.sy, w.ny);
  window_axis(w.oz, a.nz, a.W, a.g, bw, w.sz, w.nz);
  w.ex = (w.nx - 1) * a.g + bw;
  w.ey = (w.ny - 1) * a.g + bw;
  w.ez = (w.nz - 1) * a.g + bw;
  w.nc = w.nx * w.ny * w.nz;
  return w.nx > 0 && w.ny > 0 && w.nz > 0;
}

__device__ inline long long lin(const NccArgs &a, int x, int y, int z) {
  return ((long long)z * a.ny + y) * a.nx + x;
}

__device__ inline void write_block(const NccArgs &a, long long b, float best, float second,
                                   long long match, uint8_t status) {
  a.best[b] = best;
  a.second[b] = second;
  a.match[b] = (int32_t)match;
  a.status[b] = status;
}

// Shared-memory view of one staged block (raw values, as the reference reads them).
struct Staged {
  const float *x;      // base block, B floats
  const uint8_t *mb;   // base mask, B
  const float *y;      // search window, ex*ey*ez
  const uint8_t *ms;   // search mask window
  double mean_b;       // meanBase of normalizedCorrelation
};

// FP64 score of candidate (cx, cy, cz) with the reference's arithmetic:
// two sequential passes in raster order, no contraction.
template <int BW>
__device__ double exact_score(const Staged &s, const BlockWin &w, int g, int c) {
  constexpr int B = BW * BW * BW;
  int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
  const int woff = ((cz * g) * w.ey + cy * g) * w.ex + cx * g;
  double ms = 0.0;
#pragma unroll
  for (int vz = 0; vz < BW; ++vz)
#pragma unroll
    for (int vy = 0; vy < BW; ++vy)
#pragma unroll
      for (int vx = 0; vx < BW; ++vx)
        ms = __dadd_rn(ms, (double)s.y[woff + (vz * w.ey + vy) * w.ex + vx]);
  ms = __ddiv_rn(ms, (double)B);
  double prod = 0.0, bss = 0.0, sss = 0.0;
#pragma unroll
  for (int vz = 0; vz < BW; ++vz)
#pragma unroll
    for (int vy = 0; vy < BW; ++vy)
#pragma unroll
      for (int vx = 0; vx < BW; ++vx) {
        int v = (vz * BW + vy) * BW + vx;
        int wi = woff + (vz * w.ey + vy) * w.ex + vx;
        if (s.mb[v] && s.ms[wi]) {
          double bb = __dsub_rn((double)s.x[v], s.mean_b);
          double sb = __dsub_rn((double)s.y[wi], ms);
          prod = __dadd_rn(prod, __dmul_rn(bb, sb));
          bss = __dadd_rn(bss, __dmul_rn(bb, bb));
          sss = __dadd_rn(sss, __dmul_rn(sb, sb));
        }
      }
  if (bss <= 0.0 || sss <= 0.0) return -2.0;
  return __ddiv_rn(__ddiv_rn(__dmul_rn(prod, prod), bss), sss);
}

// The reference's running best / second-best update, float storage.
struct SeqTop2 {
  float best = -3.f, second = -3.f;
  int arg = -1;
  __device__ void push(double m, int c) {
    if ((double)best < m) {
      second = best;
      best = (float)m;
      arg = c;
    } else if ((double)second < m) {
      second = (float)m;
    }
  }
};

__device__ inline void top2_merge(float &a1, float &a2, float b1, float b2) {
  float m1 = fmaxf(a1, b1);
  float m2 = fmaxf(fminf(a1, b1), fmaxf(a2, b2));
  a1 = m1;
  a2 = m2;
}

__device__ inline void stage_block(const NccArgs &a, const BlockWin &w, int B, int bw, float *x,
                                   uint8_t *mb, float *y, uint8_t *ms, int &all_in_out) {
  const int tid = threadIdx.x;
  const long long obase = lin(a, w.ox, w.oy, w.oz);
  for (int v = tid; v < B; v += blockDim.x) {
    int vx = v % bw, vy = (v / bw) % bw, vz = v / (bw * bw);
    long long q = obase + ((long long)vz * a.ny + vy) * a.nx + vx;
    x[v] = __ldg(&a.base[q]);
    mb[v] = __ldg(&a.bmask[q]);
  }
  const long long wbase = lin(a, w.sx, w.sy, w.sz);
  const int nwin = w.ex * w.ey * w.ez;
  int all_in = 1;
  for (int i = tid; i < nwin; i += blockDim.x) {
    int wx = i % w.ex, wy = (i / w.ex) % w.ey, wz = i / (w.ex * w.ey);
    long long q = wbase + ((long long)wz * a.ny + wy) * a.nx + wx;
    y[i] = __ldg(&a.search[q]);
    uint8_t m = __ldg(&a.smask[q]);
    ms[i] = m;
    if (!m) all_in = 0;
  }
  all_in_out = all_in;
}

// ---------------------------------------------------------------------------
// General kernel: one CTA (128 threads) per block, any mask pattern.
// ---------------------------------------------------------------------------
template <int BW>
__global__ void __launch_bounds__(128) ncc_general_kernel(NccArgs a) {
  constexpr int B = BW * BW * BW;
  extern __shared__ __align__(16) unsigned char smem[];
  const int e3 = a.emax * a.emax * a.emax;
  const int cmax = a.W * a.W * a.W;
  float *xr = reinterpret_cast<float *>(smem);  // B raw
  float *xt = xr + B;                            // B centred (float)
  float *yw = xt + B;                            // e3
  float *sc = yw + e3;                           // cmax FP32 scores
  uint8_t *mb = reinterpret_cast<uint8_t *>(sc + cmax);
  uint8_t *mw = mb + B;
  __shared__ double s_mean;
  __shared__ float s_sxx, s_sxt;
  __shared__ int s_mball, s_cnt, s_deg[2];
  __shared__ float s_red[8];
  __shared__ int s_list[kLMax];
  __shared__ double s_ex[kLMax];
  const int tid = threadIdx.x;

  for (long long b = blockIdx.x; b < a.nblocks; b += gridDim.x) {
    __syncthreads();
    BlockWin w;
    bool ok = block_window(a, b, BW, w);
    const long long obase = lin(a, w.ox, w.oy, w.oz);
    if (a.selected && !a.selected[b]) {
      if (tid == 0) write_block(a, b, -3.f, -3.f, obase, 0);
      continue;
    }
    if (!ok) {
      if (tid == 0) write_block(a, b, -3.f, -3.f, obase, 1);
      continue;
    }
    int all_in;
    stage_block(a, w, B, BW, xr, mb, yw, mw, all_in);
    const int ms_all = __syncthreads_and(all_in);
    if (tid == 0) {
      double sum = 0.0;
      int mball = 1;
      for (int v = 0; v < B; ++v) {
        sum = __dadd_rn(sum, (double)xr[v]);
        if (!mb[v]) mball = 0;
      }
      double mean = __ddiv_rn(sum, (double)B);
      double sxx = 0.0, sxt = 0.0;
      for (int v = 0; v < B; ++v)
        if (mb[v]) {
          double d = __dsub_rn((double)xr[v], mean);
          sxx = __dadd_rn(sxx, __dmul_rn(d, d));
          sxt = __dadd_rn(sxt, d);
        }
      s_mean = mean;
      s_sxx = (float)sxx;
      s_sxt = (float)sxt;
      s_mball = mball;
      s_cnt = 0;
      s_deg[0] = s_deg[1] = -1;
    }
    __syncthreads();
    for (int v = tid; v < B; v += blockDim.x) xt[v] = (float)__dsub_rn((double)xr[v], s_mean);
    __syncthreads();
    const bool fast = s_mball && ms_all;
    const float sxx_f = s_sxx, sxt_f = s_sxt;
    // ---- stage 1: FP32 scores -------------------------------------------
    float l1 = -3.f, l2 = -3.f;
    for (int c = tid; c < w.nc; c += blockDim.x) {
      int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
      int px = w.sx + cx * a.g, py = w.sy + cy * a.g, pz = w.sz + cz * a.g;
      float2 st = __ldg(&a.stats[lin(a, px, py, pz)]);
      const float mu = st.x;
      const int woff = ((cz * a.g) * w.ey + cy * a.g) * w.ex + cx * a.g;
      float sxy = 0.f, sxx, syy;
      if (fast) {
        float acc = 0.f;
#pragma unroll
        for (int vz = 0; vz < BW; ++vz)
#pragma unroll
          for (int vy = 0; vy < BW; ++vy)
#pragma unroll
            for (int vx = 0; vx < BW; ++vx)
              acc = fmaf(xt[(vz * BW + vy) * BW + vx], yw[woff + (vz * w.ey + vy) * w.ex + vx], acc);
        sxy = acc - mu * sxt_f;
        sxx = sxx_f;
        syy = st.y;
      } else {
        float ax = 0.f, ay = 0.f;
#pragma unroll
        for (int vz = 0; vz < BW; ++vz)
#pragma unroll
          for (int vy = 0; vy < BW; ++vy)
#pragma unroll
            for (int vx = 0; vx < BW; ++vx) {
              int v = (vz * BW + vy) * BW + vx;
              int wi = woff + (vz * w.ey + vy) * w.ex + vx;
              if (mb[v] && mw[wi]) {
                float xv = xt[v];
                float d = yw[wi] - mu;
                sxy = fmaf(xv, d, sxy);
                ax = fmaf(xv, xv, ax);
                ay = fmaf(d, d, ay);
              }
            }
        sxx = ax;
        syy = s_mball ? st.y : ay;
      }
      float score = (sxx <= 0.f || syy <= 0.f) ? -2.f : (sxy * sxy) / sxx / syy;
      sc[c] = score;
      top2_merge(l1, l2, score, -3.f);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      float o1 = __shfl_down_sync(0xffffffffu, l1, off);
      float o2 = __shfl_down_sync(0xffffffffu, l2, off);
      top2_merge(l1, l2, o1, o2);
    }
    if ((tid & 31) == 0) { s_red[2 * (tid >> 5)] = l1; s_red[2 * (tid >> 5) + 1] = l2; }
    __syncthreads();
    float f1 = s_red[0], f2 = s_red[1];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) top2_merge(f1, f2, s_red[2 * k], s_red[2 * k + 1]);
    // ---- stage 2: exact refinement --------------------------------------
    const float T = f2 - 2.f * kDelta;
    for (int c = tid; c < w.nc; c += blockDim.x) {
      float s = sc[c];
      if (s > -2.f && s >= T) {
        int p = atomicAdd(&s_cnt, 1);
        if (p < kLMax) s_list[p] = c;
      }
    }
    if (f2 <= -2.f && tid == 0) {
      // fewer than two non-degenerate candidates: the first two degenerate
      // ones (in raster order) decide the second-best / the argmax
      int k = 0;
      for (int c = 0; c < w.nc && k < 2; ++c)
        if (sc[c] == -2.f) s_deg[k++] = c;
    }
    __syncthreads();
    int cnt = s_cnt;
    if (cnt > kLMax) {
      if (tid == 0) {
        unsigned int p = atomicAdd(&a.ctl[0], 1u);
        a.ovf_list[p] = (int)b;
      }
      continue;
    }
    if (tid == 0) {
      for (int k = 0; k < 2; ++k)
        if (s_deg[k] >= 0) s_list[cnt++] = s_deg[k];
      s_cnt = cnt;
    }
    __syncthreads();
    cnt = s_cnt;
    Staged sg{xr, mb, yw, mw, s_mean};
    for (int t = tid; t < cnt; t += blockDim.x) s_ex[t] = exact_score<BW>(sg, w, a.g, s_list[t]);
    __syncthreads();
    if (tid == 0) {
      // replay the sequential update in raster order
      for (int i = 1; i < cnt; ++i) {
        int ci = s_list[i];
        double ei = s_ex[i];
        int j = i - 1;
        while (j >= 0 && s_list[j] > ci) {
          s_list[j + 1] = s_list[j];
          s_ex[j + 1] = s_ex[j];
          --j;
        }
        s_list[j + 1] = ci;
        s_ex[j + 1] = ei;
      }
      SeqTop2 r;
      for (int i = 0; i < cnt; ++i) r.push(s_ex[i], s_list[i]);
      int c = r.arg < 0 ? 0 : r.arg;
      int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
      write_block(a, b, r.best, r.second,
                  lin(a, w.sx + cx * a.g, w.sy + cy * a.g, w.sz + cz * a.g), 1);
      if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)w.nc);
      atomicAdd(&a.ctl[1], (unsigned int)cnt);
    }
  }
}

// ---------------------------------------------------------------------------
// Fallback: every candidate of an overflowed block re-scored in FP64.
// ---------------------------------------------------------------------------
template <int BW>
__global__ void __launch_bounds__(128) ncc_fallback_kernel(NccArgs a) {
  constexpr int B = BW * BW * BW;
  extern __shared__ __align__(16) unsigned char smem[];
  const int e3 = a.emax * a.emax * a.emax;
  const int cmax = a.W * a.W * a.W;
  double *ex = reinterpret_cast<double *>(smem);  // cmax
  float *xr = reinterpret_cast<float *>(ex + cmax);
  float *yw = xr + B;
  uint8_t *mb = reinterpret_cast<uint8_t *>(yw + e3);
  uint8_t *mw = mb + B;
  __shared__ double s_mean;
  const int tid = threadIdx.x;
  const unsigned int n = *(volatile unsigned int *)&a.ctl[0];
  for (unsigned int i = blockIdx.x; i < n; i += gridDim.x) {
    __syncthreads();
    long long b = a.ovf_list[i];
    BlockWin w;
    block_window(a, b, BW, w);
    int all_in;
    stage_block(a, w, B, BW, xr, mb, yw, mw, all_in);
    __syncthreads();
    if (tid == 0) {
      double sum = 0.0;
      for (int v = 0; v < B; ++v) sum = __dadd_rn(sum, (double)xr[v]);
      s_mean = __ddiv_rn(sum, (double)B);
    }
    __syncthreads();
    Staged sg{xr, mb, yw, mw, s_mean};
    for (int c = tid; c < w.nc; c += blockDim.x) ex[c] = exact_score<BW>(sg, w, a.g, c);
    __syncthreads();
    if (tid < 32) {
      SeqTop2 r;
      for (int base = 0; base < w.nc; base += 32) {
        // all lanes replay the same sequence; lane 0 writes
        int lim = min(32, w.nc - base);
        for (int j = 0; j < lim; ++j) r.push(ex[base + j], base + j);
      }
      if (tid == 0) {
        int c = r.arg < 0 ? 0 : r.arg;
        int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
        write_block(a, b, r.best, r.second,
                    lin(a, w.sx + cx * a.g, w.sy + cy * a.g, w.sz + cz * a.g), 1);
        if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)w.nc);
        atomicAdd(&a.ctl[2], 1u);
      }
    }
  }
}

template <class K>
mirorr_status set_smem(K kernel, size_t smem) {
  if (smem > 48 * 1024)
    MB2_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return MIRORR_OK;
}

template <int BW>
mirorr_status launch_bw(const NccArgs &a, cudaStream_t s) {
  constexpr int B = BW * BW * BW;
  const size_t e3 = (size_t)a.emax * a.emax * a.emax, cmax = (size_t)a.W * a.W * a.W;
  size_t smem_g = sizeof(float) * (2 * B + e3 + cmax) + B + e3 + 16;
  size_t smem_f = sizeof(double) * cmax + sizeof(float) * (B + e3) + B + e3 + 16;
  if (smem_g > 200 * 1024 || smem_f > 200 * 1024) {
    set_error("search window too large for shared memory (window %d^3, %d candidates)",
              a.emax, (int)cmax);
    return MIRORR_EINVAL;
  }
  MB2_TRY(set_smem(ncc_general_kernel<BW>, smem_g));
  MB2_TRY(set_smem(ncc_fallback_kernel<BW>, smem_f));
  long long grid = a.nblocks < 148LL * 16 ? a.nblocks : 148LL * 16;
  ncc_general_kernel<BW><<<(unsigned)grid, 128, smem_g, s>>>(a);
  MB2_LAUNCH_CHECK();
  ncc_fallback_kernel<BW><<<148, 128, smem_f, s>>>(a);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace

mirorr_status launch_ncc(const BmGeom &g, const float *base, const uint8_t *bmask,
                         const float *search, const uint8_t *smask, const float2 *stats,
                         const uint8_t *selected, const BmOut &out, BmWork &w,
                         unsigned long long *ncc_count, cudaStream_t s) {
  if (g.nblocks > 0x7fffffffLL) {
    set_error("too many blocks (%lld)", g.nblocks);
    return MIRORR_EINVAL;
  }
  MB2_TRY(w.ncc_lists.ensure(sizeof(int) * (g.nblocks + 1)));
  MB2_TRY(w.ncc_ctl.ensure(sizeof(unsigned int) * 8));
  MB2_CUDA_TRY(cudaMemsetAsync(w.ncc_ctl.ptr, 0, sizeof(unsigned int) * 8, s));
  NccArgs a;
  a.base = base; a.bmask = bmask; a.search = search; a.smask = smask; a.stats = stats;
  a.selected = selected;
  a.nx = g.size[0]; a.ny = g.size[1]; a.nz = g.size[2];
  a.nbx = g.nb[0]; a.nby = g.nb[1]; a.nbz = g.nb[2];
  a.stx = g.st[0]; a.sty = g.st[1]; a.stz = g.st[2];
  a.G = g.ngap; a.g = g.bgap; a.W = g.nw;
  a.emax = (g.nw - 1) * g.bgap + g.bw;
  a.nblocks = g.nblocks;
  a.best = out.best; a.second = out.second; a.match = out.match; a.status = out.status;
  a.ncc_count = ncc_count;
  a.ovf_list = w.ncc_lists.as<int>();
  a.ctl = w.ncc_ctl.as<unsigned int>();
  switch (g.bw) {
    case 1: return launch_bw<1>(a, s);
    case 2: return launch_bw<2>(a, s);
    case 3: return launch_bw<3>(a, s);
    case 4: return launch_bw<4>(a, s);
    case 5: return launch_bw<5>(a, s);
    case 6: return launch_bw<6>(a, s);
    case 7: return launch_bw<7>(a, s);
    case 8: return launch_bw<8>(a, s);
    default:
      set_error("block width %d not supported (1..8)", g.bw);
      return MIRORR_EINVAL;
  }
}

}  // namespace mb2
