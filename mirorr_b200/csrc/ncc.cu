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
// Two stages:
//   1. FP32 search.  Every candidate is scored in FP32 (the window mean and
//      masked sum of squares come from box_stats, the base block's from
//      block_stats).  Per block the stage records the FP32 best and second
//      and the list of candidates whose FP32 score lies within 2*delta of the
//      FP32 second-best (delta bounds |FP32 - FP64|), plus the first two
//      degenerate candidates when fewer than two are non-degenerate.
//        * ncc_xlane_kernel (block width 4, window 7 or 9) and
//          ncc_warp_kernel (other widths): blocks whose base block and search
//          window are wholly inside both masks, block gap 1; cross term only,
//          one FMA per voxel and candidate.  They route the other blocks.
//        * ncc_masked_kernel: base block inside its mask, window partly
//          masked, block gap 1; three correlations.
//        * ncc_general_kernel: every other block (any mask pattern, any gap),
//          one CTA per block.
//   2. ncc_refine_kernel, one thread per block: the listed candidates are
//      re-scored in FP64 with the reference's arithmetic and summation order
//      and the sequential best/second update is replayed over them in
//      raster order.  No unlisted candidate can be the best or the second,
//      so the block's best, second and argmax equal the FP64 reference's.
//      Blocks whose list overflowed are re-scored entirely by
//      ncc_fallback_kernel.
#include <cuda.h>  // CUtensorMap (the encoder is fetched through the runtime)

#include "kernels.cuh"

namespace mb2 {

namespace {

constexpr int kK = 8;              // refinement list capacity per block
constexpr float kDelta = 1e-4f;    // bound on |FP32 score - FP64 score|

// Per-block result of the FP32 stage.
struct NccRec {
  float f1, f2;
  int cnt;        // listed candidates; -1: final result already written; > kK: overflow
  int full;       // 1: the base block and every candidate footprint lie wholly
                  // inside both masks (the refinement reads no mask)
  int32_t p[kK + 2];  // candidate origins (linear voxel index)
};

// Base-block statistics for the FP32 stage.
struct BlockStat {
  double mean;
  float sxx;   // sum over masked voxels of (x - mean)^2
  float sxt;   // sum over masked voxels of (x - mean)
  int mmode;   // base mask over the block: 1 every voxel non-zero, 2 every voxel zero, 0 mixed
  float c;     // window shift: mean of the block's own candidate footprint
};

struct NccArgs {
  const float *base;
  const uint8_t *bmask;
  const float *search;
  const uint8_t *smask;
  const float2 *stats;
  const uint8_t *selected;
  const BlockStat *bstat;
  int nx, ny, nz;
  int nbx, nby, nbz;
  int stx, sty, stz;
  int G, g, W, bw;
  int emax;
  long long nblocks;
  float *best;
  float *second;
  int32_t *match;
  uint8_t *status;
  unsigned long long *ncc_count;
  NccRec *rec;
  int *gen_list;    // [0, ctl[0]): partly masked base blocks (base-mask kernel);
                    // after nblocks + 1: partly masked windows (masked kernel)
  int *ovf_list;    // blocks for the fallback kernel
  unsigned int *ctl;  // [0] base-mask blocks, [1] overflow blocks, [2] refined candidates,
                      // [3] register-blocked blocks, [4] masked-window blocks,
                      // [5] a bounded wait on a tensor copy gave up
  const float *search_al;  // the search image with rows of spitch floats, 16-byte aligned
  int spitch;
  unsigned long long *xl_count;  // optional: candidates scored by the per-x-lane kernel
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

struct BlockWin {
  int ox, oy, oz;
  int sx, sy, sz;
  int nx, ny, nz;   // candidates per axis
  int ex, ey, ez;   // clipped window extent
  int nc;
};

__device__ inline bool block_window(const NccArgs &a, long long b, BlockWin &w) {
  int bx = (int)(b % a.nbx), by = (int)((b / a.nbx) % a.nby), bz = (int)(b / ((long long)a.nbx * a.nby));
  w.ox = a.stx + bx * a.G;
  w.oy = a.sty + by * a.G;
  w.oz = a.stz + bz * a.G;
  window_axis(w.ox, a.nx, a.W, a.g, a.bw, w.sx, w.nx);
  window_axis(w.oy, a.ny, a.W, a.g, a.bw, w.sy, w.ny);
  window_axis(w.oz, a.nz, a.W, a.g, a.bw, w.sz, w.nz);
  w.ex = (w.nx - 1) * a.g + a.bw;
  w.ey = (w.ny - 1) * a.g + a.bw;
  w.ez = (w.nz - 1) * a.g + a.bw;
  w.nc = w.nx * w.ny * w.nz;
  return w.nx > 0 && w.ny > 0 && w.nz > 0;
}

__device__ inline long long lin(const NccArgs &a, int x, int y, int z) {
  return ((long long)z * a.ny + y) * a.nx + x;
}

__device__ inline void write_final(const NccArgs &a, long long b, float best, float second,
                                   long long match, uint8_t status) {
  a.best[b] = best;
  a.second[b] = second;
  a.match[b] = (int32_t)match;
  a.status[b] = status;
}

__device__ inline void top2_merge(float &a1, float &a2, float b1, float b2) {
  float m1 = fmaxf(a1, b1);
  float m2 = fmaxf(fminf(a1, b1), fmaxf(a2, b2));
  a1 = m1;
  a2 = m2;
}

// top2_merge(a1, a2, b, -3) for a running pair with a2 >= -3.
__device__ inline void top2_push(float &a1, float &a2, float b) {
  a2 = fmaxf(a2, fminf(a1, b));
  a1 = fmaxf(a1, b);
}

__device__ inline void min2_merge(int &a1, int &a2, int b1, int b2) {
  // two smallest non-negative values of {a1, a2, b1, b2} (negative = none)
  int v[4] = {a1, a2, b1, b2};
  int m1 = -1, m2 = -1;
  for (int i = 0; i < 4; ++i) {
    int x = v[i];
    if (x < 0 || x == m1 || x == m2) continue;
    if (m1 < 0 || x < m1) { m2 = m1; m1 = x; }
    else if (m2 < 0 || x < m2) { m2 = x; }
  }
  a1 = m1;
  a2 = m2;
}

__device__ inline void cp_async4(float *dst, const float *src) {
  unsigned int d = (unsigned int)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ inline void cp_async8(void *dst, const void *src) {
  unsigned int d = (unsigned int)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
// Tensor-memory-access (TMA) load of a 3D box into shared memory, completing
// on an mbarrier (no multicast).
__device__ inline void tma_load_3d(float *dst, const CUtensorMap *map, int x, int y, int z,
                                   uint64_t *bar) {
  const unsigned int d = (unsigned int)__cvta_generic_to_shared(dst);
  const unsigned int b = (unsigned int)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(d),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(b)
      : "memory");
}
__device__ inline void mbar_init(uint64_t *bar, unsigned int count) {
  const unsigned int b = (unsigned int)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(b), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ inline void mbar_expect_tx(uint64_t *bar, unsigned int bytes) {
  const unsigned int b = (unsigned int)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(bytes)
               : "memory");
}
// Waits for phase `parity` of the barrier, at most `limit` polls; false on timeout.
__device__ inline bool mbar_wait(uint64_t *bar, unsigned int parity, int limit) {
  const unsigned int b = (unsigned int)__cvta_generic_to_shared(bar);
  for (int i = 0; i < limit; ++i) {
    unsigned int done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ inline void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// box_stats stores Syy with its sign bit set when some search-mask voxel of
// the candidate's footprint is zero.
__device__ inline bool footprint_in_mask(float syy_field) { return !signbit(syy_field); }
__device__ inline float syy_of(float syy_field) { return fabsf(syy_field); }

__device__ inline void push_deg(int &d1, int &d2, int p) {
  if (d1 < 0) d1 = p;
  else if (d2 < 0) d2 = p;
}

// A block whose base mask is zero everywhere has Sxx = 0 for every candidate,
// so every score is -2 (normalizedCorrelation's degenerate case): the
// sequential update leaves best = -2, second = -2 (-3 with one candidate) and
// the match at the first candidate in raster order, the clipped window's start.
__device__ inline void finish_unmasked_block(const NccArgs &a, long long b) {
  BlockWin w;
  if (block_window(a, b, w)) {
    write_final(a, b, -2.f, w.nc >= 2 ? -2.f : -3.f, lin(a, w.sx, w.sy, w.sz), 1);
    if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)w.nc);
  } else {
    write_final(a, b, -3.f, -3.f, lin(a, w.ox, w.oy, w.oz), 1);
  }
  a.rec[b].cnt = -1;
}

// ---------------------------------------------------------------------------
// base-block statistics (one thread per block)
// ---------------------------------------------------------------------------
// BW > 0: the block width known at compile time (the block's loads are all
// issued before the sums); BW = 0: a.bw at run time.  Same arithmetic order.
template <int BW>
__global__ void block_stat_kernel(NccArgs a) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < a.nblocks;
       b += (long long)gridDim.x * blockDim.x) {
    int bx = (int)(b % a.nbx), by = (int)((b / a.nbx) % a.nby), bz = (int)(b / ((long long)a.nbx * a.nby));
    long long o = lin(a, a.stx + bx * a.G, a.sty + by * a.G, a.stz + bz * a.G);
    const int bw = BW > 0 ? BW : a.bw;
    double sum = 0.0;
    int nin = 0;
#pragma unroll
    for (int z = 0; z < bw; ++z)
#pragma unroll
      for (int y = 0; y < bw; ++y)
#pragma unroll
        for (int x = 0; x < bw; ++x) {
          long long q = o + ((long long)z * a.ny + y) * a.nx + x;
          sum = __dadd_rn(sum, (double)__ldg(&a.base[q]));
          if (__ldg(&a.bmask[q])) ++nin;
        }
    double mean = __ddiv_rn(sum, (double)(bw * bw * bw));
    double sxx = 0.0, sxt = 0.0;
#pragma unroll
    for (int z = 0; z < bw; ++z)
#pragma unroll
      for (int y = 0; y < bw; ++y)
#pragma unroll
        for (int x = 0; x < bw; ++x) {
          long long q = o + ((long long)z * a.ny + y) * a.nx + x;
          if (__ldg(&a.bmask[q])) {
            double d = __dsub_rn((double)__ldg(&a.base[q]), mean);
            sxx = __dadd_rn(sxx, __dmul_rn(d, d));
            sxt = __dadd_rn(sxt, d);
          }
        }
    BlockStat s;
    s.mean = mean;
    s.sxx = (float)sxx;
    s.sxt = (float)sxt;
    s.mmode = nin == bw * bw * bw ? 1 : (nin == 0 ? 2 : 0);
    s.c = __ldg(&a.stats[o]).x;
    const_cast<BlockStat *>(a.bstat)[b] = s;
  }
}

// ---------------------------------------------------------------------------
// Register-blocked FP32 search for blocks whose base block lies inside its
// mask but whose window is partly masked (block gap 1).  The unmasked search
// kernels route these blocks here through the list after gen_list[nblocks].
// Several blocks per CTA; each thread owns a TY x W tile of candidates (one
// z plane) and streams window rows from shared memory.  The window is staged
// as (y - c) ms, with ms the search mask and c the mean of the block's own
// candidate (a per-block constant that keeps the FP32 cross term free of
// cancellation), and with
//   C1 = sum x~ ms (y - c),  C2 = sum x~ ms,  C3 = sum x~^2 ms,
//   Sxy = C1 - (mu - c) C2,  Sxx = C3,  Syy from box_stats
// every candidate gets C1 from the register tiles.  C2 and C3 are needed only
// where the footprint straddles the mask edge: wholly inside it they are the
// block's own sums, wholly outside it Syy = 0 and the score is -2.  Those
// candidates are listed in shared memory and finished by the whole CTA from
// per-row mask bits and per-block tables of partial sums (for each base row
// (vy, vz) and each pattern of BW mask bits along x, the sums of x~ and x~^2
// over the set bits).
// ---------------------------------------------------------------------------
template <int BW_, int W_, int TY_, int BPC_>
struct FastCfg {
  static constexpr int BW = BW_, W = W_, TY = TY_, BPC = BPC_;
  static constexpr int B = BW * BW * BW;
  static constexpr int R = W / 2;
  static constexpr int E = W + BW - 1;                 // window extent (x, z)
  static constexpr int NYG = (W + TY - 1) / TY;        // y-groups per block
  static constexpr int EY = NYG * TY + BW - 1;         // rows per plane (zero padded)
  static constexpr int EXP = (E + 3) & ~3;             // row stride (float4 aligned)
  static constexpr int Q = EY * EXP / 4;               // plane in float4 units
  static constexpr int PS = (Q + ((3 - (Q % 8)) + 8) % 8) * 4;  // plane stride, conflict-free
  static constexpr int WIN = E * PS;                   // floats per block window
  static constexpr int TPB = W * NYG;                  // threads per block
  static constexpr int NT = ((BPC * TPB + 31) / 32) * 32;
  static constexpr int NC = W * W * W;                 // candidates per block
  static constexpr int NROW = E * EY;                  // window rows per block
  static constexpr int NPAT = 1 << BW;                 // mask patterns of one base row
  static constexpr int NTAB = BW * BW * NPAT;          // table entries per block
  // dynamic shared memory, in floats: windows, base blocks, row bits, tables
  static constexpr int OFF_XT = BPC * WIN;
  static constexpr int OFF_BITS = OFF_XT + ((BPC * B + 3) & ~3);
  static constexpr int OFF_TAB = OFF_BITS + ((BPC * NROW + 3) & ~3);
  static constexpr int SMEM_FLOATS = OFF_TAB + 2 * BPC * NTAB;
  static_assert(WIN % 4 == 0 && EXP % 4 == 0 && PS % 4 == 0 && B > 0, "alignment");
  static_assert(2 * NC <= WIN, "scores and straddler list reuse the window");
  static_assert(E <= 16 && EY <= NT / 16 && NT % 32 == 0, "a window plane fits the CTA");
};

// Shared state of the per-block reduction that ends a CTA tile.
template <int BPC, int TPB>
struct TileTail {
  float red[BPC][TPB][2];
  int deg[BPC][TPB][2];
  float f[BPC][2];
  int d[BPC][2];
  int cnt[BPC];
  int list[BPC][kK];
};

// End of a CTA tile of BPC blocks: per block, the FP32 best and second and
// the first two degenerate candidates over the threads' partials (one warp
// per block), then the candidates within 2 delta of the second-best from the
// stored scores (scs: W^3 per block, -4 where not a candidate), then the
// block's record.  count_fast adds the block to the register-blocked count.
template <class C>
__device__ void finish_tile(const NccArgs &a, TileTail<C::BPC, C::TPB> &tt, const float *scs,
                            const int *s_b, const int (*s_o)[3], const int *s_state, float l1,
                            float l2, int d1, int d2, bool count_fast) {
  constexpr int BPC = C::BPC, TPB = C::TPB, TY = C::TY, W = C::W, NC = C::NC, NYG = C::NYG;
  const int tid = threadIdx.x, slot = tid / TPB, lt = tid - slot * TPB;
  const bool worker = slot < BPC;
  const bool active = worker && s_state[slot];
  const int cz = lt / NYG, cy0 = (lt - cz * NYG) * TY;
  const int nx = a.nx, ny = a.ny;
  if (worker) {
    tt.red[slot][lt][0] = l1;
    tt.red[slot][lt][1] = l2;
    tt.deg[slot][lt][0] = d1;
    tt.deg[slot][lt][1] = d2;
  }
  __syncthreads();
  {
    const int wp = tid >> 5, ln = tid & 31;
    if (wp < BPC && s_state[wp]) {
      float f1 = -3.f, f2 = -3.f;
      int e1 = -1, e2 = -1;
      for (int k = ln; k < TPB; k += 32) {
        top2_merge(f1, f2, tt.red[wp][k][0], tt.red[wp][k][1]);
        min2_merge(e1, e2, tt.deg[wp][k][0], tt.deg[wp][k][1]);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const float o1 = __shfl_down_sync(0xffffffffu, f1, off);
        const float o2 = __shfl_down_sync(0xffffffffu, f2, off);
        const int g1 = __shfl_down_sync(0xffffffffu, e1, off);
        const int g2 = __shfl_down_sync(0xffffffffu, e2, off);
        top2_merge(f1, f2, o1, o2);
        min2_merge(e1, e2, g1, g2);
      }
      if (ln == 0) {
        tt.f[wp][0] = f1;
        tt.f[wp][1] = f2;
        tt.d[wp][0] = e1;
        tt.d[wp][1] = e2;
      }
    }
  }
  __syncthreads();
  if (active) {
    const float T = tt.f[slot][1] - 2.f * kDelta;
    const int pz = s_o[slot][2] + cz;
#pragma unroll
    for (int j = 0; j < TY; ++j) {
      const int cy = cy0 + j;
      if (cy >= W) continue;
#pragma unroll
      for (int x = 0; x < W; ++x) {
        const float s = scs[slot * NC + (cz * W + cy) * W + x];
        if (s > -2.f && s >= T) {
          int pos = atomicAdd(&tt.cnt[slot], 1);
          if (pos < kK)
            tt.list[slot][pos] = (int)(((long long)pz * ny + s_o[slot][1] + cy) * nx + s_o[slot][0] + x);
        }
      }
    }
  }
  __syncthreads();
  if (active && lt == 0) {
    NccRec &rc = a.rec[s_b[slot]];
    int cnt = tt.cnt[slot];
    rc.f1 = tt.f[slot][0];
    rc.f2 = tt.f[slot][1];
    if (cnt <= kK) {
      for (int k = 0; k < cnt; ++k) rc.p[k] = tt.list[slot][k];
      if (tt.f[slot][1] <= -2.f) {
        if (tt.d[slot][0] >= 0) rc.p[cnt++] = tt.d[slot][0];
        if (tt.d[slot][1] >= 0) rc.p[cnt++] = tt.d[slot][1];
      }
    }
    rc.cnt = cnt;
    rc.full = 0;
    if (count_fast) atomicAdd(&a.ctl[3], 1u);
  }
}

template <class C>
__global__ void __launch_bounds__(C::NT, 4) ncc_masked_kernel(NccArgs a) {
  constexpr int BW = C::BW, W = C::W, TY = C::TY, BPC = C::BPC, B = C::B, R = C::R, E = C::E;
  constexpr int EY = C::EY, EXP = C::EXP, PS = C::PS, WIN = C::WIN, TPB = C::TPB, NYG = C::NYG;
  constexpr int NC = C::NC, NROW = C::NROW, NPAT = C::NPAT, NTAB = C::NTAB;
  extern __shared__ __align__(16) float sm[];
  float *win = sm;                                                // BPC * WIN: (y - c) ms
  float *xt = sm + C::OFF_XT;                                     // BPC * B: x - mu
  unsigned int *bits = reinterpret_cast<unsigned int *>(sm + C::OFF_BITS);  // BPC * NROW
  float2 *tab = reinterpret_cast<float2 *>(sm + C::OFF_TAB);      // BPC * NTAB
  // after the correlation pass the windows hold the scores and, per block,
  // the list of candidates whose footprint straddles the mask edge
  float *scs = sm;                                                // BPC * NC
  int *slist = reinterpret_cast<int *>(sm + BPC * NC);           // BPC * NC
  __shared__ TileTail<BPC, TPB> tt;
  __shared__ int s_state[BPC];           // 1 compute, 0 skip
  __shared__ int s_b[BPC];
  __shared__ int s_o[BPC][3];            // window origin (block origin - R)
  __shared__ float s_c[BPC];
  __shared__ float s_sxt[BPC];
  __shared__ float s_sxx[BPC];
  __shared__ double s_mean[BPC];
  __shared__ int s_nstr[BPC];
  const int tid = threadIdx.x;
  const int slot = tid / TPB;
  const int lt = tid - slot * TPB;
  const bool worker = slot < BPC;
  const int cz = lt / NYG;
  const int cy0 = (lt - cz * NYG) * TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long nlist = (long long)*(volatile unsigned int *)&a.ctl[4];

  for (long long base = (long long)blockIdx.x * BPC; base < nlist; base += (long long)gridDim.x * BPC) {
    __syncthreads();
    if (tid < BPC) {
      long long i = base + tid;
      int state = 0;
      tt.cnt[tid] = 0;
      if (i < nlist) {
        const int b = a.gen_list[a.nblocks + 1 + i];
        s_b[tid] = b;
        const int bx = b % a.nbx, by = (b / a.nbx) % a.nby, bz = b / (a.nbx * a.nby);
        const int ox = a.stx + bx * a.G, oy = a.sty + by * a.G, oz = a.stz + bz * a.G;
        s_o[tid][0] = ox - R;
        s_o[tid][1] = oy - R;
        s_o[tid][2] = oz - R;
        const long long o = ((long long)oz * ny + oy) * nx + ox;
        const BlockStat st = a.bstat[b];
        if (st.mmode == 1) {
          state = 1;
          s_mean[tid] = st.mean;
          s_sxt[tid] = st.sxt;
          s_sxx[tid] = st.sxx;
          s_c[tid] = __ldg(&a.stats[o]).x;  // the block's own position is a candidate
        } else {
          unsigned int p = atomicAdd(&a.ctl[0], 1u);
          a.gen_list[p] = b;
        }
      }
      s_state[tid] = state;
    }
    if (tid < BPC) s_nstr[tid] = 0;
    __syncthreads();
    // stage the windows, a 16-lane group per window row (consecutive x): the
    // E EY rows of a window (plane-major) are dealt round-robin to the CTA's
    // groups, and a group issues the loads of up to CH rows before it stores:
    // (y - c) ms, zero outside the image and in the padding, and the row's
    // mask bits (warp ballot); the base blocks as x - mu
    {
      constexpr int LPR = 16, NGRP = C::NT / LPR, RPG = (NROW + NGRP - 1) / NGRP;
      constexpr int CH = RPG < 6 ? RPG : 6;  // rows in flight per thread (registers)
      const int xl = tid & (LPR - 1), grp = tid / LPR;
      for (int s = 0; s < BPC; ++s) {
        if (!s_state[s]) continue;
        const int gx = s_o[s][0] + xl;
        const bool xin = xl < E && gx >= 0 && gx < nx;
        const float c = s_c[s];
#pragma unroll 1
        for (int i0 = 0; i0 < RPG; i0 += CH) {
          float yv[CH];
          bool msv[CH];
#pragma unroll
          for (int i = 0; i < CH; ++i) {
            const int rr = grp + (i0 + i) * NGRP, z = rr / EY, yl = rr - z * EY;
            const int gy = s_o[s][1] + yl, gz = s_o[s][2] + z;
            const bool in =
                rr < NROW && xin && yl < E && gy >= 0 && gy < ny && gz >= 0 && gz < nz;
            const long long q = ((long long)gz * ny + gy) * nx + gx;
            yv[i] = in ? __ldg(&a.search[q]) : 0.f;
            msv[i] = in && __ldg(&a.smask[q]) != 0;
          }
#pragma unroll
          for (int i = 0; i < CH; ++i) {
            const int rr = grp + (i0 + i) * NGRP, z = rr / EY, yl = rr - z * EY;
            const unsigned int bal = __ballot_sync(0xffffffffu, msv[i]);
            if (rr < NROW) {
              if (xl < EXP) win[s * WIN + z * PS + yl * EXP + xl] = msv[i] ? yv[i] - c : 0.f;
              if (xl == 0) bits[s * NROW + rr] = (bal >> (tid & LPR)) & 0xFFFFu;
            }
          }
        }
      }
    }
    for (int i = tid; i < BPC * B; i += blockDim.x) {
      const int s = i / B;
      if (!s_state[s]) continue;
      const int v = i - s * B;
      const int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
      const long long q = ((long long)(s_o[s][2] + R + vz) * ny + (s_o[s][1] + R + vy)) * nx +
                          (s_o[s][0] + R + vx);
      xt[i] = (float)__dsub_rn((double)__ldg(&a.base[q]), s_mean[s]);
    }
    __syncthreads();
    // partial-sum tables: entry (vz, vy, pattern) = sums of x~ and x~^2 over
    // the x offsets set in the pattern
    for (int i = tid; i < BPC * NTAB; i += blockDim.x) {
      const int s = i / NTAB;
      if (!s_state[s]) continue;
      const int e = i - s * NTAB;
      const int row = e / NPAT, pat = e - row * NPAT;
      const float *xr = xt + s * B + row * BW;
      float s2 = 0.f, s3 = 0.f;
#pragma unroll
      for (int vx = 0; vx < BW; ++vx)
        if ((pat >> vx) & 1) {
          s2 += xr[vx];
          s3 = fmaf(xr[vx], xr[vx], s3);
        }
      tab[i] = make_float2(s2, s3);
    }
    const bool active = worker && s_state[slot];
    float sc[TY][W];
    if (active) {
#pragma unroll
      for (int j = 0; j < TY; ++j)
#pragma unroll
        for (int x = 0; x < W; ++x) sc[j][x] = 0.f;
      const int wo = slot * WIN + cz * PS + cy0 * EXP;
      const float *tp = xt + slot * B;
#pragma unroll 1
      for (int vz = 0; vz < BW; ++vz) {
        float t[BW][BW];
#pragma unroll
        for (int vy = 0; vy < BW; ++vy)
#pragma unroll
          for (int vx = 0; vx < BW; ++vx) t[vy][vx] = tp[(vz * BW + vy) * BW + vx];
#pragma unroll
        for (int j = 0; j < TY + BW - 1; ++j) {
          float r[EXP];
          const float4 *rp = reinterpret_cast<const float4 *>(win + wo + vz * PS + j * EXP);
#pragma unroll
          for (int k = 0; k < EXP / 4; ++k) {
            const float4 q = rp[k];
            r[4 * k] = q.x; r[4 * k + 1] = q.y; r[4 * k + 2] = q.z; r[4 * k + 3] = q.w;
          }
#pragma unroll
          for (int vy = 0; vy < BW; ++vy) {
            const int jj = j - vy;
            if (jj < 0 || jj >= TY) continue;
#pragma unroll
            for (int x = 0; x < W; ++x) {
              float acc = sc[jj][x];
#pragma unroll
              for (int vx = 0; vx < BW; ++vx) acc = fmaf(t[vy][vx], r[x + vx], acc);
              sc[jj][x] = acc;
            }
          }
        }
      }
    }
    __syncthreads();  // the windows are free: scores and the straddler lists go there
    float l1 = -3.f, l2 = -3.f;
    int d1 = -1, d2 = -1;
    if (active) {
      const float sxt = s_sxt[slot], sxx_b = s_sxx[slot], cc = s_c[slot];
      const int pz = s_o[slot][2] + cz;
#pragma unroll
      for (int j = 0; j < TY; ++j) {
        const int cy = cy0 + j;
        if (cy >= W) continue;
        const int py = s_o[slot][1] + cy;
        const bool rowok = py >= 0 && py <= ny - BW && pz >= 0 && pz <= nz - BW;
        const long long prow = ((long long)pz * ny + py) * nx + s_o[slot][0];
#pragma unroll
        for (int x = 0; x < W; ++x) {
          const int px = s_o[slot][0] + x;
          const int cl = (cz * W + cy) * W + x;
          float s = -4.f;  // not a candidate
          if (rowok && px >= 0 && px <= nx - BW) {
            const float2 st = __ldg(&a.stats[prow + x]);
            const float syy = syy_of(st.y);
            if (syy <= 0.f) {
              s = -2.f;
            } else if (footprint_in_mask(st.y)) {
              const float sxy = sc[j][x] - (st.x - cc) * sxt;
              s = sxx_b <= 0.f ? -2.f : __fdividef(__fdividef(sxy * sxy, sxx_b), syy);
            } else {
              // footprint across the mask edge: C1 kept, finished below
              slist[slot * NC + atomicAdd(&s_nstr[slot], 1)] = cl;
              scs[slot * NC + cl] = sc[j][x];
              continue;
            }
            if (s == -2.f) push_deg(d1, d2, (int)(prow + x));
            top2_merge(l1, l2, s, -3.f);
          }
          scs[slot * NC + cl] = s;
        }
      }
    }
    __syncthreads();
    if (active) {
      // this block's straddling candidates: C2 and C3 from the row bits and
      // the tables
      const int nstr = s_nstr[slot];
      const unsigned int *rb = bits + slot * NROW;
      const float2 *tb = tab + slot * NTAB;
      const float cc = s_c[slot];
      for (int i = lt; i < nstr; i += TPB) {
        const int cl = slist[slot * NC + i];
        const int x = cl % W, cy = (cl / W) % W, czz = cl / (W * W);
        float c2 = 0.f, c3 = 0.f;
#pragma unroll
        for (int vz = 0; vz < BW; ++vz)
#pragma unroll
          for (int vy = 0; vy < BW; ++vy) {
            const unsigned int pat = (rb[(czz + vz) * EY + cy + vy] >> x) & (NPAT - 1);
            const float2 q = tb[(vz * BW + vy) * NPAT + pat];
            c2 += q.x;
            c3 += q.y;
          }
        const long long p = ((long long)(s_o[slot][2] + czz) * ny + s_o[slot][1] + cy) * nx +
                            s_o[slot][0] + x;
        const float2 st = __ldg(&a.stats[p]);
        const float sxy = scs[slot * NC + cl] - (st.x - cc) * c2;
        const float s = c3 <= 0.f ? -2.f : __fdividef(__fdividef(sxy * sxy, c3), syy_of(st.y));
        scs[slot * NC + cl] = s;
        if (s == -2.f) min2_merge(d1, d2, (int)p, -1);  // list order: keep the two smallest
        top2_merge(l1, l2, s, -3.f);
      }
    }
    finish_tile<C>(a, tt, scs, s_b, s_o, s_state, l1, l2, d1, d2, true);
  }
}

// ---------------------------------------------------------------------------
// Register-blocked FP32 search for blocks whose base block is partly masked
// (block gap 1); the unmasked search kernels route them here through
// gen_list[0 .. ctl[0]).  With m = mb ms (base and search mask), mu the
// unmasked mean of the candidate footprint and x~ = x - mean of the base
// block:
//   Sxy = sum m x~ (y - mu),  Sxx = sum m x~^2,  Syy = sum m (y - mu)^2,
// each summed directly (no expansion around a constant, so no cancellation).
// The window is staged as y ms and ms, the base block as (mb x~, mb x~^2, mb);
// per candidate voxel, md = ms (y - mu) is one FMA and the three sums take
// one FMA each plus a multiply for mb md.  Tile layout as the masked kernel.
// ---------------------------------------------------------------------------
template <class C>
__global__ void __launch_bounds__(C::NT, 2) ncc_basemask_kernel(NccArgs a) {
  constexpr int BW = C::BW, W = C::W, TY = C::TY, BPC = C::BPC, B = C::B, R = C::R, E = C::E;
  constexpr int EY = C::EY, EXP = C::EXP, PS = C::PS, WIN = C::WIN, TPB = C::TPB, NYG = C::NYG;
  constexpr int NC = C::NC;
  extern __shared__ __align__(16) float sm[];
  float *win = sm;                                               // BPC * WIN: y ms
  float *mwin = sm + BPC * WIN;                                  // BPC * WIN: ms
  float4 *xb = reinterpret_cast<float4 *>(sm + 2 * BPC * WIN);  // BPC * B: mb x~, mb x~^2, mb
  float *scs = sm;  // after the correlation pass: BPC * NC scores
  __shared__ TileTail<BPC, TPB> tt;
  __shared__ int s_state[BPC];
  __shared__ int s_b[BPC];
  __shared__ int s_o[BPC][3];
  __shared__ double s_mean[BPC];
  const int tid = threadIdx.x;
  const int slot = tid / TPB;
  const int lt = tid - slot * TPB;
  const bool worker = slot < BPC;
  const int cz = lt / NYG;
  const int cy0 = (lt - cz * NYG) * TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long nlist = (long long)*(volatile unsigned int *)&a.ctl[0];

  for (long long base = (long long)blockIdx.x * BPC; base < nlist; base += (long long)gridDim.x * BPC) {
    __syncthreads();
    if (tid < BPC) {
      long long i = base + tid;
      int state = 0;
      tt.cnt[tid] = 0;
      if (i < nlist) {
        const int b = a.gen_list[i];
        s_b[tid] = b;
        const int bx = b % a.nbx, by = (b / a.nbx) % a.nby, bz = b / (a.nbx * a.nby);
        s_o[tid][0] = a.stx + bx * a.G - R;
        s_o[tid][1] = a.sty + by * a.G - R;
        s_o[tid][2] = a.stz + bz * a.G - R;
        const BlockStat st = a.bstat[b];
        if (st.mmode == 2) {
          finish_unmasked_block(a, b);
        } else {
          state = 1;
          s_mean[tid] = st.mean;
        }
      }
      s_state[tid] = state;
    }
    __syncthreads();
    // stage the windows one plane per pass, a 16-lane group per window row:
    // y ms and ms, zero outside the image and in the padding
    {
      constexpr int LPR = 16;
      const int xl = tid & (LPR - 1), yl = tid / LPR;
      const long long plane = (long long)nx * ny;
      for (int s = 0; s < BPC; ++s) {
        if (!s_state[s]) continue;
        const int gx = s_o[s][0] + xl, gy = s_o[s][1] + yl, gz0 = s_o[s][2];
        const bool xyin = xl < E && yl < E && gx >= 0 && gy >= 0 && gx < nx && gy < ny;
        const long long q0 = ((long long)gz0 * ny + gy) * nx + gx;
        float *wd = win + s * WIN + yl * EXP + xl;
        float *md = mwin + s * WIN + yl * EXP + xl;
        if (yl < EY && xl < EXP) {
#pragma unroll
          for (int z = 0; z < E; ++z) {
            const int gz = gz0 + z;
            const bool in = xyin && gz >= 0 && gz < nz;
            const long long q = q0 + z * plane;
            const float yv = in ? __ldg(&a.search[q]) : 0.f;
            const bool ms = in && __ldg(&a.smask[q]) != 0;
            wd[z * PS] = ms ? yv : 0.f;
            md[z * PS] = ms ? 1.f : 0.f;
          }
        }
      }
    }
    for (int i = tid; i < BPC * B; i += blockDim.x) {
      const int s = i / B;
      if (!s_state[s]) continue;
      const int v = i - s * B;
      const int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
      const long long q = ((long long)(s_o[s][2] + R + vz) * ny + (s_o[s][1] + R + vy)) * nx +
                          (s_o[s][0] + R + vx);
      const float xv = (float)__dsub_rn((double)__ldg(&a.base[q]), s_mean[s]);
      const float mb = __ldg(&a.bmask[q]) ? 1.f : 0.f;
      xb[i] = make_float4(mb * xv, mb * (xv * xv), mb, 0.f);
    }
    __syncthreads();
    const bool active = worker && s_state[slot];
    float s1[TY][W], s2[TY][W], s3[TY][W], nmu[TY][W];
    if (active) {
      const int pz = s_o[slot][2] + cz;
#pragma unroll
      for (int j = 0; j < TY; ++j)
#pragma unroll
        for (int x = 0; x < W; ++x) {
          const int py = s_o[slot][1] + cy0 + j, px = s_o[slot][0] + x;
          const bool ok = cy0 + j < W && px >= 0 && px <= nx - BW && py >= 0 && py <= ny - BW &&
                          pz >= 0 && pz <= nz - BW;
          nmu[j][x] = ok ? -__ldg(&a.stats[((long long)pz * ny + py) * nx + px]).x : 0.f;
          s1[j][x] = 0.f;
          s2[j][x] = 0.f;
          s3[j][x] = 0.f;
        }
      const int wo = slot * WIN + cz * PS + cy0 * EXP;
      const float4 *tp = xb + slot * B;
#pragma unroll 1
      for (int vz = 0; vz < BW; ++vz) {
#pragma unroll
        for (int j = 0; j < TY + BW - 1; ++j) {
          float r[EXP], m[EXP];
          const float4 *rp = reinterpret_cast<const float4 *>(win + wo + vz * PS + j * EXP);
          const float4 *mp = reinterpret_cast<const float4 *>(mwin + wo + vz * PS + j * EXP);
#pragma unroll
          for (int k = 0; k < EXP / 4; ++k) {
            const float4 q = rp[k], u = mp[k];
            r[4 * k] = q.x; r[4 * k + 1] = q.y; r[4 * k + 2] = q.z; r[4 * k + 3] = q.w;
            m[4 * k] = u.x; m[4 * k + 1] = u.y; m[4 * k + 2] = u.z; m[4 * k + 3] = u.w;
          }
#pragma unroll
          for (int vy = 0; vy < BW; ++vy) {
            const int jj = j - vy;
            if (jj < 0 || jj >= TY) continue;
            // the base row (vy, vz), read where it is used (fewer live registers)
            float4 t[BW];
#pragma unroll
            for (int vx = 0; vx < BW; ++vx) t[vx] = tp[(vz * BW + vy) * BW + vx];
#pragma unroll
            for (int x = 0; x < W; ++x) {
              float a1 = s1[jj][x], a2 = s2[jj][x], a3 = s3[jj][x];
#pragma unroll
              for (int vx = 0; vx < BW; ++vx) {
                const float md = fmaf(nmu[jj][x], m[x + vx], r[x + vx]);  // ms (y - mu)
                a1 = fmaf(t[vx].x, md, a1);
                a2 = fmaf(t[vx].y, m[x + vx], a2);
                a3 = fmaf(t[vx].z * md, md, a3);
              }
              s1[jj][x] = a1;
              s2[jj][x] = a2;
              s3[jj][x] = a3;
            }
          }
        }
      }
    }
    __syncthreads();  // the windows are free: the scores go there
    float l1 = -3.f, l2 = -3.f;
    int d1 = -1, d2 = -1;
    if (active) {
      const int pz = s_o[slot][2] + cz;
#pragma unroll
      for (int j = 0; j < TY; ++j) {
        const int cy = cy0 + j;
        if (cy >= W) continue;
        const int py = s_o[slot][1] + cy;
        const bool rowok = py >= 0 && py <= ny - BW && pz >= 0 && pz <= nz - BW;
        const long long prow = ((long long)pz * ny + py) * nx + s_o[slot][0];
#pragma unroll
        for (int x = 0; x < W; ++x) {
          const int px = s_o[slot][0] + x;
          float s = -4.f;  // not a candidate
          if (rowok && px >= 0 && px <= nx - BW) {
            const float sxy = s1[j][x], sxx = s2[j][x], syy = s3[j][x];
            s = (sxx <= 0.f || syy <= 0.f) ? -2.f : __fdividef(__fdividef(sxy * sxy, sxx), syy);
            if (s == -2.f) push_deg(d1, d2, (int)(prow + x));
            top2_merge(l1, l2, s, -3.f);
          }
          scs[slot * NC + (cz * W + cy) * W + x] = s;
        }
      }
    }
    finish_tile<C>(a, tt, scs, s_b, s_o, s_state, l1, l2, d1, d2, false);
  }
}

// ---------------------------------------------------------------------------
// Warp-level register-blocked FP32 search for blocks whose base block and
// window are wholly inside both masks (block gap 1).  Each warp holds SPW
// blocks (one per LPS = 32/SPW lanes) and runs independently of the other
// warps of its CTA (no CTA barrier): stage the window rows and the base
// block with asynchronous copies, score a TY x W tile of candidates per lane
// (one z plane, cross term only) streaming window rows from shared memory,
// reduce with shuffles, emit the block's refinement list.  The window is
// staged as y - c (c: mean of the block's own candidate), so
// Sxy = sum x~ (y - c) - (mu - c) sum x~ has no FP32 cancellation.  Blocks
// with a partly masked window go to the masked kernel, blocks with a partly
// masked base block to the base-mask kernel.
// ---------------------------------------------------------------------------
template <int BW_, int W_, int TY_, int SPW_, int WPC_, int MINB_>
struct WarpCfg {
  static constexpr int BW = BW_, W = W_, TY = TY_, SPW = SPW_;
  static constexpr int MINB = MINB_;                   // resident CTAs per SM aimed for
  static constexpr int LPS = 32 / SPW;                 // lanes per block
  static constexpr int B = BW * BW * BW;
  static constexpr int R = W / 2;
  static constexpr int E = W + BW - 1;
  static constexpr int NYG = (W + TY - 1) / TY;
  static constexpr int TPB = W * NYG;                  // working lanes per block
  static constexpr int EY = NYG * TY + BW - 1;
  static constexpr int EXP = (E + 3) & ~3;
  static constexpr int Q = EY * EXP / 4;
  static constexpr int PS = (Q + ((3 - (Q % 8)) + 8) % 8) * 4;
  static constexpr int WIN = E * PS;
  static constexpr int NSTAT = W * W * W;             // candidate statistics (float2)
  // floats per block slot; a multiple of 4 keeps every slot's window rows
  // 16-byte aligned for the float4 row loads
  static constexpr int SLOT = (WIN + ((B + 3) & ~3) + 2 * NSTAT + 3) & ~3;
  static_assert(SLOT % 4 == 0 && WIN % 4 == 0 && EXP % 4 == 0 && PS % 4 == 0, "alignment");
  static constexpr int WPC = WPC_;                     // warps per CTA
  static_assert(TPB <= LPS, "tile does not fit the lanes of a block");
};

template <class C>
__global__ void __launch_bounds__(C::WPC * 32, C::MINB) ncc_warp_kernel(NccArgs a) {
  constexpr int BW = C::BW, W = C::W, TY = C::TY, SPW = C::SPW, LPS = C::LPS, B = C::B;
  constexpr int R = C::R, E = C::E, NYG = C::NYG, TPB = C::TPB, EY = C::EY, EXP = C::EXP;
  constexpr int PS = C::PS, WIN = C::WIN, SLOT = C::SLOT, WPC = C::WPC;
  extern __shared__ __align__(16) float sm[];
  __shared__ int s_cnt[WPC * SPW];
  __shared__ int s_list[WPC * SPW][kK];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sl = lane / LPS, sln = lane - sl * LPS;
  const int slot = warp * SPW + sl;
  float *win = sm + slot * SLOT;
  float *xt = win + WIN;
  float2 *sst = reinterpret_cast<float2 *>(xt + ((B + 3) & ~3));  // W^3 candidate statistics
  const bool worker = sln < TPB;
  const int cz = sln / NYG;
  const int cy0 = (sln - cz * NYG) * TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const unsigned full = 0xffffffffu;
  const int src = sl * LPS;
  const unsigned seg = (LPS == 32) ? full : (((1u << LPS) - 1u) << src);
  const long long stride = (long long)gridDim.x * WPC * SPW;

  for (long long base = ((long long)blockIdx.x * WPC + warp) * SPW; base < a.nblocks; base += stride) {
    const long long bl = base + sl;
    const bool valid = bl < a.nblocks;
    const int b = valid ? (int)bl : 0;
    // ---- set-up: every lane of the block reads the same statistics --------
    const BlockStat st = a.bstat[b];
    const int bx = b % a.nbx, by = (b / a.nbx) % a.nby, bz = b / (a.nbx * a.nby);
    const int bx0 = a.stx + bx * a.G, by0 = a.sty + by * a.G, bz0 = a.stz + bz * a.G;
    const int ox = bx0 - R, oy = by0 - R, oz = bz0 - R;
    int state = 0;
    if (valid) {
      // with block gap 1 every window holds at least the block's own origin
      const bool sel = !a.selected || a.selected[b];
      if (!sel) {
        if (sln == 0) {
          write_final(a, b, -3.f, -3.f, ((long long)bz0 * ny + by0) * nx + bx0, 0);
          a.rec[b].cnt = -1;
        }
      } else if (st.mmode == 1) {
        state = 1;
      } else if (sln == 0) {
        if (st.mmode == 2) {
          finish_unmasked_block(a, b);
        } else {
          unsigned int p = atomicAdd(&a.ctl[0], 1u);
          a.gen_list[p] = b;
        }
      }
    }
    if (sln == 0) s_cnt[slot] = 0;
    const float cc = st.c;
    // ---- staging: coalesced asynchronous copies (x fastest across lanes) ---
    if (state) {
      for (int e = sln; e < E * EY * E; e += LPS) {
        const int row = e / E, x = e - row * E;
        const int z = row / EY, y = row - z * EY;
        const int gx = ox + x, gy = oy + y, gz = oz + z;
        float *dst = win + z * PS + y * EXP + x;
        if (y < E && gx >= 0 && gy >= 0 && gz >= 0 && gx < nx && gy < ny && gz < nz)
          cp_async4(dst, a.search + ((long long)gz * ny + gy) * nx + gx);
        else
          *dst = 0.f;
      }
      for (int v = sln; v < B; v += LPS) {
        const int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
        cp_async4(xt + v, a.base + ((long long)(bz0 + vz) * ny + (by0 + vy)) * nx + (bx0 + vx));
      }
      for (int e = sln; e < W * W * W; e += LPS) {
        const int row = e / W, x = e - row * W;
        const int z = row / W, y = row - z * W;
        const int gx = ox + x, gy = oy + y, gz = oz + z;
        if (gx >= 0 && gy >= 0 && gz >= 0 && gx <= nx - BW && gy <= ny - BW && gz <= nz - BW)
          cp_async8(sst + e, a.stats + ((long long)gz * ny + gy) * nx + gx);
        else
          sst[e] = make_float2(__int_as_float(0x7fc00000), 0.f);  // not a candidate (NaN)
      }
    }
    cp_async_wait_all();
    __syncwarp();
    // partly masked window -> masked kernel
    bool inmask = true;
    if (state) {
      for (int e = sln; e < W * W * W; e += LPS) {
        const float2 q = sst[e];
        if (q.x == q.x && !footprint_in_mask(q.y)) inmask = false;
      }
    }
    const unsigned bad = __ballot_sync(full, !inmask);
    if (state && (bad & seg)) {
      if (sln == 0) {
        unsigned int p = atomicAdd(&a.ctl[4], 1u);
        a.gen_list[a.nblocks + 1 + p] = b;
      }
      state = 0;
    }
    if (state) {
      for (int r = sln; r < E * EY; r += LPS) {
        const int z = r / EY, y = r - z * EY;
        float4 *p4 = reinterpret_cast<float4 *>(win + z * PS + y * EXP);
#pragma unroll
        for (int k = 0; k < EXP / 4; ++k) {
          float4 q = p4[k];
          q.x -= cc; q.y -= cc; q.z -= cc; q.w -= cc;
          p4[k] = q;
        }
      }
      for (int v = sln; v < B; v += LPS) xt[v] = (float)__dsub_rn((double)xt[v], st.mean);
    }
    __syncwarp();
    // ---- FP32 scores of the lane's tile -----------------------------------
    float sc[TY][W];
    float l1 = -3.f, l2 = -3.f;
    int d1 = -1, d2 = -1;
    const bool active = state && worker;
    if (active) {
#pragma unroll
      for (int j = 0; j < TY; ++j)
#pragma unroll
        for (int x = 0; x < W; ++x) sc[j][x] = 0.f;
      const float *wp = win + cz * PS + cy0 * EXP;
#pragma unroll 1
      for (int vz = 0; vz < BW; ++vz) {
        float t[BW][BW];
#pragma unroll
        for (int vy = 0; vy < BW; ++vy)
#pragma unroll
          for (int vx = 0; vx < BW; ++vx) t[vy][vx] = xt[(vz * BW + vy) * BW + vx];
#pragma unroll
        for (int j = 0; j < TY + BW - 1; ++j) {
          float r[EXP];
          const float4 *rp = reinterpret_cast<const float4 *>(wp + vz * PS + j * EXP);
#pragma unroll
          for (int k = 0; k < EXP / 4; ++k) {
            float4 q = rp[k];
            r[4 * k] = q.x; r[4 * k + 1] = q.y; r[4 * k + 2] = q.z; r[4 * k + 3] = q.w;
          }
#pragma unroll
          for (int vy = 0; vy < BW; ++vy) {
            const int jj = j - vy;
            if (jj < 0 || jj >= TY) continue;
#pragma unroll
            for (int x = 0; x < W; ++x) {
              float acc = sc[jj][x];
#pragma unroll
              for (int vx = 0; vx < BW; ++vx) acc = fmaf(t[vy][vx], r[x + vx], acc);
              sc[jj][x] = acc;
            }
          }
        }
      }
      const float sxt = st.sxt, sxx_b = st.sxx;
#pragma unroll
      for (int j = 0; j < TY; ++j) {
        const int cy = cy0 + j;
#pragma unroll
        for (int x = 0; x < W; ++x) {
          float s = -4.f;  // not a candidate
          if (cy < W) {
            const float2 q = sst[(cz * W + cy) * W + x];
            if (q.x == q.x) {
              const float syy = syy_of(q.y);
              const float sxy = sc[j][x] - (q.x - cc) * sxt;
              s = (sxx_b <= 0.f || syy <= 0.f) ? -2.f : __fdividef(__fdividef(sxy * sxy, sxx_b), syy);
              if (s == -2.f) push_deg(d1, d2, (int)(((long long)(oz + cz) * ny + oy + cy) * nx + ox + x));
              top2_merge(l1, l2, s, -3.f);
            }
          }
          sc[j][x] = s;
        }
      }
    }
    // ---- block-level reduction (within the block's lanes) -----------------
#pragma unroll
    for (int off = LPS / 2; off > 0; off >>= 1) {
      float o1 = __shfl_down_sync(full, l1, off, LPS);
      float o2 = __shfl_down_sync(full, l2, off, LPS);
      int e1 = __shfl_down_sync(full, d1, off, LPS);
      int e2 = __shfl_down_sync(full, d2, off, LPS);
      top2_merge(l1, l2, o1, o2);
      min2_merge(d1, d2, e1, e2);
    }
    const float f1 = __shfl_sync(full, l1, src), f2 = __shfl_sync(full, l2, src);
    d1 = __shfl_sync(full, d1, src);
    d2 = __shfl_sync(full, d2, src);
    if (active) {
      const float T = f2 - 2.f * kDelta;
#pragma unroll
      for (int j = 0; j < TY; ++j)
#pragma unroll
        for (int x = 0; x < W; ++x) {
          const float s = sc[j][x];
          if (s > -2.f && s >= T) {
            const int pos = atomicAdd(&s_cnt[slot], 1);
            if (pos < kK)
              s_list[slot][pos] = (int)(((long long)(oz + cz) * ny + oy + cy0 + j) * nx + ox + x);
          }
        }
    }
    __syncwarp();
    if (state && sln == 0) {
      NccRec &rc = a.rec[b];
      int cnt = s_cnt[slot];
      rc.f1 = f1;
      rc.f2 = f2;
      if (cnt <= kK) {
        for (int k = 0; k < cnt; ++k) rc.p[k] = s_list[slot][k];
        if (f2 <= -2.f) {
          if (d1 >= 0) rc.p[cnt++] = d1;
          if (d2 >= 0) rc.p[cnt++] = d2;
        }
      }
      rc.cnt = cnt;
      rc.full = 1;
      atomicAdd(&a.ctl[3], 1u);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Window-AND of the footprint flags, per block: wand[b] is 1 when every
// candidate of block b's window whose footprint lies inside the volume has its
// footprint wholly inside the search mask (box_stats: Syy sign bit clear).
// Separable, evaluated only at the blocks' window starts: along x for every
// (y, z) row, then along y and z at block resolution; out-of-range positions
// count as 1.
// ---------------------------------------------------------------------------
__global__ void wand_x_kernel(const float2 *stats, uint8_t *out, int nx, int ny, int nz, int nbx,
                              int stx, int G, int W, int bw) {
  const int R = W / 2;
  const long long n = (long long)nbx * ny * nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(i % nbx);
    const long long yz = i / nbx;
    const int y = (int)(yz % ny), z = (int)(yz / ny);
    const int sx = stx + bx * G - R;
    unsigned v = 1;
    if (y <= ny - bw && z <= nz - bw) {
      const float *fy = reinterpret_cast<const float *>(stats + yz * nx) + 1;
      for (int q = sx < 0 ? 0 : sx; q < sx + W && q <= nx - bw; ++q)
        v &= footprint_in_mask(__ldg(fy + 2 * q)) ? 1u : 0u;
    }
    out[i] = (uint8_t)v;
  }
}

// [outer][n][inner] -> [outer][nb][inner]: AND over the window of W starting
// at st + b G - R along the middle axis.
__global__ void wand_axis_kernel(const uint8_t *in, uint8_t *out, long long inner, int n,
                                 long long outer, int nb, int st, int G, int W) {
  const int R = W / 2;
  const long long total = outer * nb * inner;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long ii = i % inner;
    const long long r = i / inner;
    const int sa = st + (int)(r % nb) * G - R;
    const long long o = r / nb;
    unsigned v = 1;
    for (int q = sa < 0 ? 0 : sa; q < sa + W && q < n; ++q) v &= in[(o * n + q) * inner + ii];
    out[i] = (uint8_t)v;
  }
}

// ---------------------------------------------------------------------------
// Lane-per-x-offset FP32 search, block width 4, block gap 1, for blocks whose
// base block and window lie wholly inside both masks.
//
// A CTA of NW warps (NL = 32 NW lanes) takes BPW = NL / W consecutive blocks
// of one row of the block grid (same by, bz); with two warps and W = 9 that
// is 7 blocks on 63 of 64 lanes.  Lane (k, x) scores the W x W candidates of
// block k whose x offset in the window is x, i.e. every (cy, cz).  The
// blocks' windows overlap along x, so the CTA stages their union once: one tensor (TMA) copy
// of an rpu x E x E box from a 16-byte aligned x, zero-filled outside the
// volume, completing on an mbarrier whose wait is bounded; at every load the
// lanes read consecutive floats of one row (no bank conflicts).  The lane's base
// block (x~ = x - mean, 64 values) sits in registers and each window row is
// read once, shifted by the block's constant c as it is read
// (Sxy = sum x~ (y - c) - (mu - c) sum x~ keeps the FP32 cross term free of
// cancellation).  A window plane wz feeds the candidate planes wz - 3 .. wz;
// their accumulators rotate through four register sets and a plane is scored
// once its last window plane has been read.  The scores go to the shared
// memory of a window plane every warp has consumed (a CTA barrier per plane
// makes sure of it; lanes without a block run the loop on placeholder data
// and write nothing); after the block-level top-2
// reduction one pass over them lists the candidates within 2 delta of the
// block's FP32 second-best.  Blocks whose window is partly masked (window-AND
// of the footprint flags) go to the masked kernel, blocks with a partly
// masked base block to the base-mask kernel.
// ---------------------------------------------------------------------------
constexpr int kXWarpsPerSM = 12;  // resident warps per SM aimed for
constexpr int kXWarps = 2;        // warps per CTA

struct XArgs {
  const uint8_t *wand;  // per block: window wholly inside the search mask
  int rpu;              // union row pitch in floats (multiple of 4, the box's x extent)
  int nch;              // 16-byte chunks per union row
  int tpr;              // warp tiles per row of the block grid
  long long ntiles;
};

template <int W, int NW>
__global__ void __launch_bounds__(32 * NW, kXWarpsPerSM / NW)
    ncc_xlane_kernel(NccArgs a, XArgs xa, const __grid_constant__ CUtensorMap tmap) {
  constexpr int R = W / 2, E = W + 3, NL = 32 * NW, BPW = NL / W;
  extern __shared__ __align__(16) float sm[];
  __shared__ __align__(8) uint64_t s_bar;
  // the tensor copy's destination starts on 128 bytes (the allocation has 128 spare)
  float *const sma = reinterpret_cast<float *>(
      sm + ((128u - ((unsigned int)__cvta_generic_to_shared(sm) & 127u)) & 127u) / sizeof(float));
  float *win = sma;                     // E * E * rpu
  float *xt = sma + E * E * xa.rpu;     // BPW * 64
  float2 *qbuf = reinterpret_cast<float2 *>(xt + BPW * 64);  // NL * W
  __shared__ float s_red[BPW][W][2];
  __shared__ int s_deg[BPW][W][2];
  __shared__ float s_f[BPW][2];
  __shared__ int s_cnt[BPW];
  __shared__ int s_list[BPW][kK];
  const int lane = threadIdx.x;
  const int k = lane / W, x = lane - k * W;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  if (lane == 0) mbar_init(&s_bar, 1);
  __syncthreads();
  unsigned int phase = 0;
  const unsigned int win_bytes = (unsigned int)(E * E * xa.rpu * sizeof(float));

  for (long long tile = blockIdx.x; tile < xa.ntiles; tile += gridDim.x) {
    const long long grow = tile / xa.tpr;
    const int bx0 = (int)(tile - grow * xa.tpr) * BPW;
    const int by = (int)(grow % a.nby), bz = (int)(grow / a.nby);
    const int nbt = min(BPW, a.nbx - bx0);
    const bool mine = k < nbt;
    const long long brow = ((long long)bz * a.nby + by) * a.nbx;
    const long long b = brow + bx0 + (mine ? k : 0);
    const int oy = a.sty + by * a.G - R, oz = a.stz + bz * a.G - R;
    const int ox0 = a.stx + bx0 * a.G - R;
    const int ox = ox0 + k * a.G;
    const int xu = ox0 & ~3;             // union origin, rounded down to 16 bytes
    // ---- routing ----------------------------------------------------------
    int state = 0;
    BlockStat st;
    st.mean = 0.0; st.sxx = 0.f; st.sxt = 0.f; st.mmode = 0; st.c = 0.f;
    if (mine) {
      st = a.bstat[b];
      const bool sel = !a.selected || a.selected[b];
      if (!sel) {
        if (x == 0) {
          write_final(a, b, -3.f, -3.f, lin(a, ox + R, oy + R, oz + R), 0);
          a.rec[b].cnt = -1;
        }
      } else if (st.mmode == 1) {
        state = 1;
      } else if (x == 0) {
        if (st.mmode == 2) {
          finish_unmasked_block(a, b);
        } else {
          unsigned int p = atomicAdd(&a.ctl[0], 1u);
          a.gen_list[p] = (int)b;
        }
      }
    }
    if (lane < BPW) s_cnt[lane] = 0;
    // ---- window inside the search mask? -----------------------------------
    const int px = ox + x;
    const bool xok = px >= 0 && px <= nx - 4;
    unsigned yok = 0;
#pragma unroll
    for (int cy = 0; cy < W; ++cy)
      if (oy + cy >= 0 && oy + cy <= ny - 4) yok |= 1u << cy;
    // a partly masked window sends the block (all of its lanes read the same
    // flag) to the masked kernel
    if (state && !xa.wand[b]) {
      if (x == 0) {
        unsigned int p = atomicAdd(&a.ctl[4], 1u);
        a.gen_list[a.nblocks + 1 + p] = (int)b;
      }
      state = 0;
    }
    if (!__syncthreads_or(state)) continue;
    // ---- staging: the union window by one tensor copy (zero outside the
    // volume), the base blocks (x~) by the lanes meanwhile --------------------
    const int rpu = xa.rpu;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier reads of win
    __syncthreads();
    if (lane == 0) {
      mbar_expect_tx(&s_bar, win_bytes);
      tma_load_3d(win, &tmap, xu, oy, oz, &s_bar);
    }
    for (int i = lane; i < nbt * 64; i += NL) {
      const int kk = i >> 6, v = i & 63;
      const int vx = v & 3, vy = (v >> 2) & 3, vz = v >> 4;
      const long long q = ((long long)(oz + R + vz) * ny + (oy + R + vy)) * nx +
                          (ox0 + kk * a.G + R + vx);
      const double mk = a.bstat[brow + bx0 + kk].mean;
      xt[i] = (float)__dsub_rn((double)__ldg(&a.base[q]), mk);
    }
    // the give-up decision is the CTA's, so no thread is left at a barrier
    const bool landed = mbar_wait(&s_bar, phase, 1 << 22);
    if (__syncthreads_or(!landed)) {
      if (lane == 0) atomicExch(&a.ctl[5], 1u);
      return;
    }
    phase ^= 1u;
    __syncthreads();
    // ---- FP32 scores ---------------------------------------------------------
    float l1 = -3.f, l2 = -3.f;
    int d1 = -1, d2 = -1;
    const int E_rpu = E * rpu;
    {
      // every thread runs the plane loop (it holds CTA barriers); a lane
      // without a block computes on its own placeholder data and writes nothing
      const bool real = state != 0;
      float t[64];
      const float4 *tp = reinterpret_cast<const float4 *>(xt + (real ? k : 0) * 64);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float4 q = tp[i];
        t[4 * i] = q.x; t[4 * i + 1] = q.y; t[4 * i + 2] = q.z; t[4 * i + 3] = q.w;
      }
      const float c = st.c, sxt = st.sxt, sxx = st.sxx;
      const float rsxx = sxx > 0.f ? 1.f / sxx : 0.f;
      float2 *qb = qbuf + lane * W;
      const float2 *st0 = a.stats + (((long long)oz * ny + oy) * nx + px);
      const float *rp = win + (real ? ox - xu : 0) + x;
      // acc[j]: candidate plane cz = wz - 3 + j.  Window plane wz feeds the
      // planes wz - 3 .. wz (j = 3 - vz); planes outside 0 .. W-1, fed at the
      // first and last three window planes, are never scored.
      float acc[4][W];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int cy = 0; cy < W; ++cy) acc[j][cy] = 0.f;
#pragma unroll 1
      for (int wz = 0; wz < E; ++wz) {
        const int cz = wz - 3;
        const bool zok = real && cz >= 0 && xok && oz + cz >= 0 && oz + cz <= nz - 4;
        if (zok) {
          // statistics of the plane completed below, fetched meanwhile
#pragma unroll
          for (int cy = 0; cy < W; ++cy)
            if ((yok >> cy) & 1u) cp_async8(qb + cy, st0 + ((long long)cz * ny + cy) * nx);
          asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
#pragma unroll
        for (int wy = 0; wy < E; ++wy) {
          float r[4];
#pragma unroll
          for (int vx = 0; vx < 4; ++vx) r[vx] = rp[vx] - c;
          rp += rpu;
#pragma unroll
          for (int vx = 0; vx < 4; ++vx)
#pragma unroll
            for (int vz = 0; vz < 4; ++vz)
#pragma unroll
              for (int vy = 0; vy < 4; ++vy) {
                const int cy = wy - vy;
                if (cy < 0 || cy >= W) continue;
                acc[3 - vz][cy] = fmaf(t[(vz * 4 + vy) * 4 + vx], r[vx], acc[3 - vz][cy]);
              }
        }
        if (cz >= 0) {
          // window plane cz was read three planes ago by every warp: its rows
          // now hold the scores of candidate plane cz (lane-major, W per lane)
          __syncthreads();
          if (zok) {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            float *sc = win + cz * E_rpu + lane * W;
            const long long prow = ((long long)(oz + cz) * ny + oy) * nx + px;
#pragma unroll
            for (int cy = 0; cy < W; ++cy) {
              if (!((yok >> cy) & 1u)) continue;
              const float2 q = qb[cy];
              const float sxy = acc[0][cy] - (q.x - c) * sxt;
              const float s = (sxx <= 0.f || q.y <= 0.f) ? -2.f : __fdividef(sxy * sxy * rsxx, q.y);
              top2_push(l1, l2, s);
              if (s == -2.f) push_deg(d1, d2, (int)(prow + (long long)cy * nx));
              sc[cy] = s;
            }
          }
        }
        // rotate: plane wz - 3 is done, plane wz + 1 starts
#pragma unroll
        for (int cy = 0; cy < W; ++cy) {
          acc[0][cy] = acc[1][cy];
          acc[1][cy] = acc[2][cy];
          acc[2][cy] = acc[3][cy];
          acc[3][cy] = 0.f;
        }
      }
    }
    // ---- block-level reduction and refinement list --------------------------
    if (state) {
      s_red[k][x][0] = l1; s_red[k][x][1] = l2;
      s_deg[k][x][0] = d1; s_deg[k][x][1] = d2;
    }
    __syncthreads();
    if (state && x == 0) {
      float f1 = -3.f, f2 = -3.f;
      int e1 = -1, e2 = -1;
      for (int j = 0; j < W; ++j) {
        top2_merge(f1, f2, s_red[k][j][0], s_red[k][j][1]);
        min2_merge(e1, e2, s_deg[k][j][0], s_deg[k][j][1]);
      }
      s_f[k][0] = f1; s_f[k][1] = f2;
      s_deg[k][0][0] = e1; s_deg[k][0][1] = e2;
    }
    __syncthreads();
    if (state && xok) {
      // candidates within 2 delta of the block's FP32 second-best
      const float T2 = s_f[k][1] - 2.f * kDelta;
      for (int cz = 0; cz < W; ++cz) {
        if (oz + cz < 0 || oz + cz > nz - 4) continue;
        const float *sc = win + cz * E_rpu + lane * W;
        const long long prow = ((long long)(oz + cz) * ny + oy) * nx + px;
#pragma unroll
        for (int cy = 0; cy < W; ++cy) {
          if (!((yok >> cy) & 1u)) continue;
          const float sv = sc[cy];
          if (sv > -2.f && sv >= T2) {
            const int pos = atomicAdd(&s_cnt[k], 1);
            if (pos < kK) s_list[k][pos] = (int)(prow + (long long)cy * nx);
          }
        }
      }
    }
    __syncthreads();
    if (state && x == 0) {
      NccRec &rc = a.rec[b];
      const float f1 = s_f[k][0], f2 = s_f[k][1];
      int cnt = s_cnt[k];
      rc.f1 = f1;
      rc.f2 = f2;
      if (cnt <= kK) {
        for (int j = 0; j < cnt; ++j) rc.p[j] = s_list[k][j];
        if (f2 <= -2.f) {
          if (s_deg[k][0][0] >= 0) rc.p[cnt++] = s_deg[k][0][0];
          if (s_deg[k][0][1] >= 0) rc.p[cnt++] = s_deg[k][0][1];
        }
      }
      rc.cnt = cnt;
      rc.full = 1;
      atomicAdd(&a.ctl[3], 1u);
      if (a.xl_count) {
        // candidates of the clipped window: valid offsets per axis
        auto nval = [](int o, int n) {
          const int lo = o < 0 ? -o : 0, hi = min(W - 1, n - 4 - o);
          return hi >= lo ? hi - lo + 1 : 0;
        };
        atomicAdd(a.xl_count, (unsigned long long)nval(ox, nx) * nval(oy, ny) * nval(oz, nz));
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// General FP32 search: one CTA (128 threads) per block, any mask pattern and
// block gap, for geometries without the register-blocked kernels.
// ---------------------------------------------------------------------------
template <int BW>
__global__ void __launch_bounds__(128) ncc_general_kernel(NccArgs a) {
  constexpr int B = BW * BW * BW;
  extern __shared__ __align__(16) unsigned char smem[];
  const int e3 = a.emax * a.emax * a.emax;
  float *xt = reinterpret_cast<float *>(smem);  // B centred (float)
  float *yw = xt + B;                            // e3
  float *scs = yw + e3;                          // W^3 candidate scores
  uint8_t *mb = reinterpret_cast<uint8_t *>(scs + a.W * a.W * a.W);
  uint8_t *mw = mb + B;
  __shared__ int s_cnt, s_list[kK];
  __shared__ float s_red[4][2];
  __shared__ int s_deg[4][2];
  const int tid = threadIdx.x;

  for (long long b = blockIdx.x; b < a.nblocks; b += gridDim.x) {
    __syncthreads();
    BlockWin w;
    bool ok = block_window(a, b, w);
    const long long obase = lin(a, w.ox, w.oy, w.oz);
    if (a.selected && !a.selected[b]) {
      if (tid == 0) { write_final(a, b, -3.f, -3.f, obase, 0); a.rec[b].cnt = -1; }
      continue;
    }
    if (!ok) {
      if (tid == 0) { write_final(a, b, -3.f, -3.f, obase, 1); a.rec[b].cnt = -1; }
      continue;
    }
    const BlockStat bst = a.bstat[b];
    if (bst.mmode == 2) {
      if (tid == 0) finish_unmasked_block(a, b);
      continue;
    }
    for (int v = tid; v < B; v += blockDim.x) {
      int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
      long long q = obase + ((long long)vz * a.ny + vy) * a.nx + vx;
      xt[v] = (float)__dsub_rn((double)__ldg(&a.base[q]), bst.mean);
      mb[v] = __ldg(&a.bmask[q]);
    }
    const long long wbase = lin(a, w.sx, w.sy, w.sz);
    const int nwin = w.ex * w.ey * w.ez;
    int all_in = 1;
    for (int k = tid; k < nwin; k += blockDim.x) {
      int wx = k % w.ex, wy = (k / w.ex) % w.ey, wz = k / (w.ex * w.ey);
      long long q = wbase + ((long long)wz * a.ny + wy) * a.nx + wx;
      yw[k] = __ldg(&a.search[q]);
      uint8_t m = __ldg(&a.smask[q]);
      mw[k] = m;
      if (!m) all_in = 0;
    }
    if (tid == 0) s_cnt = 0;
    const int ms_all = __syncthreads_and(all_in);
    const bool fast = bst.mmode == 1 && ms_all;
    float l1 = -3.f, l2 = -3.f;
    int d1 = -1, d2 = -1;
    // pass 0 scores every candidate (FP32 top-2, first degenerate candidates);
    // pass 1 lists those within 2 delta of the second-best from the stored scores
    for (int pass = 0; pass < 2; ++pass) {
      float T = 0.f;
      if (pass == 1) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          float o1 = __shfl_down_sync(0xffffffffu, l1, off);
          float o2 = __shfl_down_sync(0xffffffffu, l2, off);
          int e1 = __shfl_down_sync(0xffffffffu, d1, off);
          int e2 = __shfl_down_sync(0xffffffffu, d2, off);
          top2_merge(l1, l2, o1, o2);
          min2_merge(d1, d2, e1, e2);
        }
        if ((tid & 31) == 0) {
          s_red[tid >> 5][0] = l1; s_red[tid >> 5][1] = l2;
          s_deg[tid >> 5][0] = d1; s_deg[tid >> 5][1] = d2;
        }
        __syncthreads();
        l1 = s_red[0][0]; l2 = s_red[0][1]; d1 = s_deg[0][0]; d2 = s_deg[0][1];
        for (int k = 1; k < 4; ++k) {
          top2_merge(l1, l2, s_red[k][0], s_red[k][1]);
          min2_merge(d1, d2, s_deg[k][0], s_deg[k][1]);
        }
        T = l2 - 2.f * kDelta;
      }
      for (int c = tid; c < w.nc; c += blockDim.x) {
        int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
        int px = w.sx + cx * a.g, py = w.sy + cy * a.g, pz = w.sz + cz * a.g;
        long long p = lin(a, px, py, pz);
        if (pass == 1) {
          const float s = scs[c];
          if (s > -2.f && s >= T) {
            int pos = atomicAdd(&s_cnt, 1);
            if (pos < kK) s_list[pos] = (int)p;
          }
          continue;
        }
        float2 st = __ldg(&a.stats[p]);
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
          sxy = acc - mu * bst.sxt;
          sxx = bst.sxx;
          syy = syy_of(st.y);
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
          syy = bst.mmode == 1 ? syy_of(st.y) : ay;
        }
        float s = (sxx <= 0.f || syy <= 0.f) ? -2.f : (sxy * sxy) / sxx / syy;
        top2_merge(l1, l2, s, -3.f);
        if (s == -2.f) push_deg(d1, d2, (int)p);
        scs[c] = s;
      }
    }
    __syncthreads();
    if (tid == 0) {
      NccRec &rc = a.rec[b];
      int cnt = s_cnt;
      rc.f1 = l1;
      rc.f2 = l2;
      if (cnt <= kK) {
        for (int k = 0; k < cnt; ++k) rc.p[k] = s_list[k];
        if (l2 <= -2.f) {
          if (d1 >= 0) rc.p[cnt++] = d1;
          if (d2 >= 0) rc.p[cnt++] = d2;
        }
      }
      rc.cnt = cnt;
      rc.full = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 refinement: one thread per block.
// ---------------------------------------------------------------------------
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

// normalizedCorrelation in FP64 with the reference's summation order.
template <int BW>
__device__ double exact_score(const NccArgs &a, const float *x, const uint8_t *mb, double mean_b,
                              long long p) {
  constexpr int B = BW * BW * BW;
  double ms = 0.0;
  for (int vz = 0; vz < BW; ++vz)
    for (int vy = 0; vy < BW; ++vy)
#pragma unroll
      for (int vx = 0; vx < BW; ++vx)
        ms = __dadd_rn(ms, (double)__ldg(&a.search[p + ((long long)vz * a.ny + vy) * a.nx + vx]));
  ms = __ddiv_rn(ms, (double)B);
  double prod = 0.0, bss = 0.0, sss = 0.0;
  for (int vz = 0; vz < BW; ++vz)
    for (int vy = 0; vy < BW; ++vy)
#pragma unroll
      for (int vx = 0; vx < BW; ++vx) {
        const int v = (vz * BW + vy) * BW + vx;
        const long long q = p + ((long long)vz * a.ny + vy) * a.nx + vx;
        if (mb[v] && __ldg(&a.smask[q])) {
          double bb = __dsub_rn((double)x[v], mean_b);
          double sb = __dsub_rn((double)__ldg(&a.search[q]), ms);
          prod = __dadd_rn(prod, __dmul_rn(bb, sb));
          bss = __dadd_rn(bss, __dmul_rn(bb, bb));
          sss = __dadd_rn(sss, __dmul_rn(sb, sb));
        }
      }
  if (bss <= 0.0 || sss <= 0.0) return -2.0;
  return __ddiv_rn(__ddiv_rn(__dmul_rn(prod, prod), bss), sss);
}

template <int BW>
__global__ void __launch_bounds__(128) ncc_refine_kernel(NccArgs a) {
  constexpr int B = BW * BW * BW;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < a.nblocks;
       b += (long long)gridDim.x * blockDim.x) {
    NccRec rc = a.rec[b];
    if (rc.cnt < 0) continue;
    if (rc.cnt > kK) {
      unsigned int pos = atomicAdd(&a.ctl[1], 1u);
      a.ovf_list[pos] = (int)b;
      continue;
    }
    BlockWin w;
    block_window(a, b, w);
    const long long o = lin(a, w.ox, w.oy, w.oz);
    // raster order = increasing linear index
    int n = rc.cnt;
    for (int i = 1; i < n; ++i) {
      int v = rc.p[i], j = i - 1;
      while (j >= 0 && rc.p[j] > v) { rc.p[j + 1] = rc.p[j]; --j; }
      rc.p[j + 1] = v;
    }
    SeqTop2 r;
    if constexpr (B <= 64) {
      // every voxel of the base block and of a candidate loaded into
      // registers first (all loads in flight at once), then the reference's
      // FP64 chains in raster order
      // the thread's base block in a transposed shared slice (conflict-free)
      __shared__ float xs[B][128];
      const long long plane = (long long)a.ny * a.nx;
      // with both masks full over the block's footprints every mask bit is
      // set: no mask is read
      const bool full = rc.full == 1;
      constexpr unsigned long long kAll = B == 64 ? ~0ULL : (1ULL << B) - 1ULL;
      unsigned long long mbm = full ? kAll : 0ULL;
      {
        float x[B];
#pragma unroll
        for (int v = 0; v < B; ++v) {
          const int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
          const long long q = o + vz * plane + (long long)vy * a.nx + vx;
          x[v] = __ldg(&a.base[q]);
          if (!full && __ldg(&a.bmask[q])) mbm |= 1ULL << v;
        }
#pragma unroll
        for (int v = 0; v < B; ++v) xs[v][threadIdx.x] = x[v];
      }
      double sum = 0.0;
#pragma unroll
      for (int v = 0; v < B; ++v) sum = __dadd_rn(sum, (double)xs[v][threadIdx.x]);
      const double mean_b = __ddiv_rn(sum, (double)B);
      for (int i = 0; i < n; ++i) {
        const long long p = rc.p[i];
        float y[B];
        unsigned long long msm = full ? kAll : 0ULL;
#pragma unroll
        for (int v = 0; v < B; ++v) {
          const int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
          const long long q = p + vz * plane + (long long)vy * a.nx + vx;
          y[v] = __ldg(&a.search[q]);
          if (!full && __ldg(&a.smask[q])) msm |= 1ULL << v;
        }
        double ms = 0.0;
#pragma unroll
        for (int v = 0; v < B; ++v) ms = __dadd_rn(ms, (double)y[v]);
        ms = __ddiv_rn(ms, (double)B);
        const unsigned long long m = mbm & msm;
        double prod = 0.0, bss = 0.0, sss = 0.0;
#pragma unroll
        for (int v = 0; v < B; ++v) {
          if ((m >> v) & 1ULL) {
            const double bb = __dsub_rn((double)xs[v][threadIdx.x], mean_b);
            const double sb = __dsub_rn((double)y[v], ms);
            prod = __dadd_rn(prod, __dmul_rn(bb, sb));
            bss = __dadd_rn(bss, __dmul_rn(bb, bb));
            sss = __dadd_rn(sss, __dmul_rn(sb, sb));
          }
        }
        const double sc = (bss <= 0.0 || sss <= 0.0)
                              ? -2.0 : __ddiv_rn(__ddiv_rn(__dmul_rn(prod, prod), bss), sss);
        r.push(sc, (int)p);
      }
    } else {
      float x[B];
      uint8_t mb[B];
      double sum = 0.0;
      for (int vz = 0; vz < BW; ++vz)
        for (int vy = 0; vy < BW; ++vy)
#pragma unroll
          for (int vx = 0; vx < BW; ++vx) {
            const int v = (vz * BW + vy) * BW + vx;
            const long long q = o + ((long long)vz * a.ny + vy) * a.nx + vx;
            x[v] = __ldg(&a.base[q]);
            mb[v] = __ldg(&a.bmask[q]);
            sum = __dadd_rn(sum, (double)x[v]);
          }
      const double mean_b = __ddiv_rn(sum, (double)B);
      for (int i = 0; i < n; ++i) r.push(exact_score<BW>(a, x, mb, mean_b, rc.p[i]), rc.p[i]);
    }
    write_final(a, b, r.best, r.second, r.arg < 0 ? lin(a, w.sx, w.sy, w.sz) : r.arg, 1);
    if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)w.nc);
    atomicAdd(&a.ctl[2], (unsigned int)n);
  }
}

// ---------------------------------------------------------------------------
// Fallback: every candidate of an overflowed block re-scored in FP64.
// ---------------------------------------------------------------------------
template <int BW>
__global__ void __launch_bounds__(128) ncc_fallback_kernel(NccArgs a) {
  constexpr int B = BW * BW * BW;
  extern __shared__ __align__(16) unsigned char smem[];
  double *ex = reinterpret_cast<double *>(smem);  // W^3
  __shared__ float xs[B];
  __shared__ uint8_t mbs[B];
  __shared__ double s_mean;
  const int tid = threadIdx.x;
  const unsigned int n = *(volatile unsigned int *)&a.ctl[1];
  for (unsigned int i = blockIdx.x; i < n; i += gridDim.x) {
    __syncthreads();
    const long long b = a.ovf_list[i];
    BlockWin w;
    block_window(a, b, w);
    const long long o = lin(a, w.ox, w.oy, w.oz);
    for (int v = tid; v < B; v += blockDim.x) {
      int vx = v % BW, vy = (v / BW) % BW, vz = v / (BW * BW);
      long long q = o + ((long long)vz * a.ny + vy) * a.nx + vx;
      xs[v] = __ldg(&a.base[q]);
      mbs[v] = __ldg(&a.bmask[q]);
    }
    __syncthreads();
    if (tid == 0) {
      double sum = 0.0;
      for (int v = 0; v < B; ++v) sum = __dadd_rn(sum, (double)xs[v]);
      s_mean = __ddiv_rn(sum, (double)B);
    }
    __syncthreads();
    for (int c = tid; c < w.nc; c += blockDim.x) {
      int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
      ex[c] = exact_score<BW>(a, xs, mbs, s_mean,
                              lin(a, w.sx + cx * a.g, w.sy + cy * a.g, w.sz + cz * a.g));
    }
    __syncthreads();
    if (tid == 0) {
      SeqTop2 r;
      for (int c = 0; c < w.nc; ++c) r.push(ex[c], c);
      int c = r.arg < 0 ? 0 : r.arg;
      int cx = c % w.nx, cy = (c / w.nx) % w.ny, cz = c / (w.nx * w.ny);
      write_final(a, b, r.best, r.second, lin(a, w.sx + cx * a.g, w.sy + cy * a.g, w.sz + cz * a.g), 1);
      if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)w.nc);
    }
  }
}

template <class K>
mirorr_status set_smem(K kernel, size_t smem) {
  MB2_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return MIRORR_OK;
}

template <class C>
mirorr_status launch_masked(const NccArgs &a, cudaStream_t s) {
  size_t smem = sizeof(float) * (size_t)C::SMEM_FLOATS;
  MB2_TRY(set_smem(ncc_masked_kernel<C>, smem));
  long long need = (a.nblocks + C::BPC - 1) / C::BPC;
  long long grid = need < (long long)sm_count() * 8 ? need : (long long)sm_count() * 8;
  ncc_masked_kernel<C><<<(unsigned)grid, C::NT, smem, s>>>(a);
  MB2_LAUNCH_CHECK();
  // then the blocks with a partly masked base block (the list grows in both
  // kernels above)
  const size_t smem_b = sizeof(float) * (size_t)C::BPC * (2 * C::WIN + 4 * C::B);
  MB2_TRY(set_smem(ncc_basemask_kernel<C>, smem_b));
  const long long grid_b = need < (long long)sm_count() * 4 ? need : (long long)sm_count() * 4;
  ncc_basemask_kernel<C><<<(unsigned)grid_b, C::NT, smem_b, s>>>(a);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

template <class CW>
mirorr_status launch_warp(const NccArgs &a, cudaStream_t s) {
  size_t smem = sizeof(float) * (size_t)CW::WPC * CW::SPW * CW::SLOT;
  MB2_TRY(set_smem(ncc_warp_kernel<CW>, smem));
  long long need = (a.nblocks + CW::WPC * CW::SPW - 1) / (CW::WPC * CW::SPW);
  long long grid = need < (long long)sm_count() * CW::MINB * 4 ? need : (long long)sm_count() * CW::MINB * 4;
  ncc_warp_kernel<CW><<<(unsigned)grid, CW::WPC * 32, smem, s>>>(a);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

template <class CW, class CM>
mirorr_status launch_fast(const NccArgs &a, cudaStream_t s) {
  MB2_TRY((launch_warp<CW>(a, s)));
  MB2_TRY((launch_masked<CM>(a, s)));
  return MIRORR_OK;
}

template <int BW>
mirorr_status launch_rest(const NccArgs &a, bool all_general, cudaStream_t s) {
  constexpr int B = BW * BW * BW;
  const size_t e3 = (size_t)a.emax * a.emax * a.emax, cmax = (size_t)a.W * a.W * a.W;
  size_t smem_g = sizeof(float) * (B + e3 + cmax) + B + e3 + 16;
  size_t smem_f = sizeof(double) * cmax + 16;
  if (smem_g > 200 * 1024 || smem_f > 200 * 1024) {
    set_error("search window too large for shared memory (window %d^3, %d candidates)",
              a.emax, (int)cmax);
    return MIRORR_EINVAL;
  }
  MB2_TRY(set_smem(ncc_general_kernel<BW>, smem_g));
  MB2_TRY(set_smem(ncc_fallback_kernel<BW>, smem_f));
  if (all_general) {
    // no register-blocked kernels for this geometry: every block here
    long long grid = a.nblocks < (long long)sm_count() * 16 ? a.nblocks : (long long)sm_count() * 16;
    ncc_general_kernel<BW><<<(unsigned)grid, 128, smem_g, s>>>(a);
    MB2_LAUNCH_CHECK();
  }
  long long rgrid = (a.nblocks + 127) / 128;
  ncc_refine_kernel<BW><<<(unsigned)rgrid, 128, 0, s>>>(a);
  MB2_LAUNCH_CHECK();
  ncc_fallback_kernel<BW><<<(unsigned)sm_count(), 128, smem_f, s>>>(a);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

// Per-x-lane search (block width 4) and the masked-window kernel; done is
// false when the union window would not fit (very wide block spacing).
// cuTensorMapEncodeTiled, fetched once through the runtime (no -lcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  }
  return fn;
}

template <int W, class CM>
mirorr_status launch_xlane(NccArgs &a, BmWork &w, cudaStream_t s, bool &done,
                           cudaEvent_t *kev) {
  constexpr int E = W + 3, NL = 32 * kXWarps, BPW = NL / W;
  done = false;
  const long long u = (long long)(BPW - 1) * a.G + E;   // union row length
  XArgs xa;
  xa.nch = (int)((u + 6) / 4);
  xa.rpu = 4 * xa.nch;
  // each window plane must hold one plane of scores (W per lane) once read
  const int min_rpu = ((BPW * W * W + E - 1) / E + 3) & ~3;
  if (xa.rpu < min_rpu) {
    xa.rpu = min_rpu;
    xa.nch = min_rpu / 4;
  }
  xa.tpr = (a.nbx + BPW - 1) / BPW;
  xa.ntiles = (long long)xa.tpr * a.nby * a.nbz;
  const size_t smem = sizeof(float) * ((size_t)E * E * xa.rpu + BPW * 64 + 2 * NL * W) + 128;
  if (xa.rpu > 256 || smem > 64 * 1024) return MIRORR_OK;  // tensor box limit
  // rows of the search image must start on 16 bytes for the 16-byte copies
  a.search_al = a.search;
  a.spitch = a.nx;
  if ((a.nx & 3) || (reinterpret_cast<uintptr_t>(a.search) & 15)) {
    a.spitch = (a.nx + 3) & ~3;
    MB2_TRY(w.ncc_pad.ensure(sizeof(float) * (size_t)a.spitch * a.ny * a.nz));
    MB2_CUDA_TRY(cudaMemcpy2DAsync(w.ncc_pad.ptr, sizeof(float) * a.spitch, a.search,
                                   sizeof(float) * a.nx, sizeof(float) * a.nx,
                                   (size_t)a.ny * a.nz, cudaMemcpyDeviceToDevice, s));
    a.search_al = w.ncc_pad.as<float>();
  }
  // window-AND of the footprint flags per block, one pass per axis
  {
    const size_t n1 = (size_t)a.nbx * a.ny * a.nz, n2 = (size_t)a.nbx * a.nby * a.nz;
    MB2_TRY(w.ncc_wand.ensure(n1 + n2 + (size_t)a.nblocks));
    uint8_t *b1 = w.ncc_wand.as<uint8_t>(), *b2 = b1 + n1, *b3 = b2 + n2;
    const unsigned g = (unsigned)sm_count() * 8;
    wand_x_kernel<<<g, 256, 0, s>>>(a.stats, b1, a.nx, a.ny, a.nz, a.nbx, a.stx, a.G, W, 4);
    MB2_LAUNCH_CHECK();
    wand_axis_kernel<<<g, 256, 0, s>>>(b1, b2, a.nbx, a.ny, a.nz, a.nby, a.sty, a.G, W);
    MB2_LAUNCH_CHECK();
    wand_axis_kernel<<<g, 256, 0, s>>>(b2, b3, (long long)a.nbx * a.nby, a.nz, 1, a.nbz, a.stz,
                                       a.G, W);
    MB2_LAUNCH_CHECK();
    xa.wand = b3;
  }
  // tensor map of the search image: x extent nx (zero beyond), rows of spitch floats
  CUtensorMap tmap;
  {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) {
      set_error("cuTensorMapEncodeTiled is not available from the driver");
      return MIRORR_ECUDA;
    }
    const cuuint64_t gdim[3] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz};
    const cuuint64_t gstride[2] = {(cuuint64_t)a.spitch * sizeof(float),
                                   (cuuint64_t)a.spitch * a.ny * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)xa.rpu, (cuuint32_t)E, (cuuint32_t)E};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(a.search_al),
                     gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
      return MIRORR_ECUDA;
    }
  }
  MB2_TRY(set_smem(ncc_xlane_kernel<W, kXWarps>, smem));
  const long long kCtas = (long long)sm_count() * (kXWarpsPerSM / kXWarps);
  const long long grid = xa.ntiles < kCtas ? xa.ntiles : kCtas;
  if (kev) MB2_CUDA_TRY(cudaEventRecord(kev[0], s));
  ncc_xlane_kernel<W, kXWarps><<<(unsigned)grid, NL, smem, s>>>(a, xa, tmap);
  MB2_LAUNCH_CHECK();
  if (kev) MB2_CUDA_TRY(cudaEventRecord(kev[1], s));
  MB2_TRY((launch_masked<CM>(a, s)));
  done = true;
  return MIRORR_OK;
}

// Block width / window combinations with a register-blocked fast kernel.
bool run_fast(NccArgs &a, BmWork &w, cudaStream_t s, mirorr_status &st, cudaEvent_t *kev,
              bool &xl_ran) {
  xl_ran = false;
  if (a.g != 1) return false;
  if ((long long)a.nx * a.ny * a.nz >= (1LL << 31)) return false;
  if (a.bw == 4 && a.W == 9) {
    bool done = false;
    st = launch_xlane<9, FastCfg<4, 9, 1, 3>>(a, w, s, done, kev);
    xl_ran = done;
    if (st != MIRORR_OK || done) return true;
    st = launch_fast<WarpCfg<4, 9, 3, 1, 5, 3>, FastCfg<4, 9, 1, 3>>(a, s);
    return true;
  }
  if (a.bw == 4 && a.W == 7) {
    bool done = false;
    st = launch_xlane<7, FastCfg<4, 7, 1, 5>>(a, w, s, done, kev);
    xl_ran = done;
    if (st != MIRORR_OK || done) return true;
    st = launch_fast<WarpCfg<4, 7, 4, 2, 4, 3>, FastCfg<4, 7, 1, 5>>(a, s);
    return true;
  }
  if (a.bw == 5 && a.W == 11) {
    st = launch_fast<WarpCfg<5, 11, 6, 1, 4, 2>, FastCfg<5, 11, 1, 2>>(a, s);
    return true;
  }
  return false;
}

}  // namespace

mirorr_status launch_ncc(const BmGeom &g, const float *base, const uint8_t *bmask,
                         const float *search, const uint8_t *smask, const float2 *stats,
                         const uint8_t *selected, const BmOut &out, BmWork &w,
                         unsigned long long *ncc_count, cudaStream_t s, cudaEvent_t *kev,
                         unsigned long long *xl_count, bool *xl_ran) {
  if (g.nblocks > 0x7fffffffLL) {
    set_error("too many blocks (%lld)", g.nblocks);
    return MIRORR_EINVAL;
  }
  MB2_TRY(w.ncc_lists.ensure(sizeof(int) * 3 * (g.nblocks + 1)));
  const void *ctl_before = w.ncc_ctl.ptr;
  MB2_TRY(w.ncc_ctl.ensure(sizeof(unsigned int) * 8));
  MB2_TRY(w.ncc_rec.ensure(sizeof(NccRec) * g.nblocks));
  MB2_TRY(w.ncc_bstat.ensure(sizeof(BlockStat) * g.nblocks));
  // counters 0..4 restart every call; [5] (a bounded wait gave up) stays set
  // until the host reads it (ncc_take_timeout)
  MB2_CUDA_TRY(cudaMemsetAsync(w.ncc_ctl.ptr, 0,
                               sizeof(unsigned int) * (w.ncc_ctl.ptr == ctl_before ? 5 : 8), s));
  NccArgs a;
  a.base = base; a.bmask = bmask; a.search = search; a.smask = smask; a.stats = stats;
  a.selected = selected;
  a.bstat = w.ncc_bstat.as<BlockStat>();
  a.nx = g.size[0]; a.ny = g.size[1]; a.nz = g.size[2];
  a.nbx = g.nb[0]; a.nby = g.nb[1]; a.nbz = g.nb[2];
  a.stx = g.st[0]; a.sty = g.st[1]; a.stz = g.st[2];
  a.G = g.ngap; a.g = g.bgap; a.W = g.nw; a.bw = g.bw;
  a.emax = (g.nw - 1) * g.bgap + g.bw;
  a.nblocks = g.nblocks;
  a.best = out.best; a.second = out.second; a.match = out.match; a.status = out.status;
  a.ncc_count = ncc_count;
  a.rec = w.ncc_rec.as<NccRec>();
  a.gen_list = w.ncc_lists.as<int>();
  a.ovf_list = a.gen_list + 2 * (g.nblocks + 1);
  a.ctl = w.ncc_ctl.as<unsigned int>();
  a.search_al = search;
  a.spitch = g.size[0];
  a.xl_count = xl_count;
  {
    long long grid = (g.nblocks + 127) / 128;
    if (grid > (long long)sm_count() * 16) grid = (long long)sm_count() * 16;
    if (a.bw == 4) block_stat_kernel<4><<<(unsigned)grid, 128, 0, s>>>(a);
    else if (a.bw == 5) block_stat_kernel<5><<<(unsigned)grid, 128, 0, s>>>(a);
    else block_stat_kernel<0><<<(unsigned)grid, 128, 0, s>>>(a);
    MB2_LAUNCH_CHECK();
  }
  mirorr_status st = MIRORR_OK;
  bool ran = false;
  bool fast = run_fast(a, w, s, st, kev, ran);
  if (xl_ran) *xl_ran = ran;
  MB2_TRY(st);
  switch (g.bw) {
    case 1: return launch_rest<1>(a, !fast, s);
    case 2: return launch_rest<2>(a, !fast, s);
    case 3: return launch_rest<3>(a, !fast, s);
    case 4: return launch_rest<4>(a, !fast, s);
    case 5: return launch_rest<5>(a, !fast, s);
    case 6: return launch_rest<6>(a, !fast, s);
    case 7: return launch_rest<7>(a, !fast, s);
    case 8: return launch_rest<8>(a, !fast, s);
    default:
      set_error("block width %d not supported (1..8)", g.bw);
      return MIRORR_EINVAL;
  }
}

mirorr_status launch_window_and(const BmGeom &g, const float2 *stats, DevBuf &buf,
                                const uint8_t **wand, cudaStream_t s) {
  const int nx = g.size[0], ny = g.size[1], nz = g.size[2];
  const size_t n1 = (size_t)g.nb[0] * ny * nz, n2 = (size_t)g.nb[0] * g.nb[1] * nz;
  MB2_TRY(buf.ensure(n1 + n2 + (size_t)g.nblocks));
  uint8_t *b1 = buf.as<uint8_t>(), *b2 = b1 + n1, *b3 = b2 + n2;
  const unsigned grid = (unsigned)sm_count() * 8;
  wand_x_kernel<<<grid, 256, 0, s>>>(stats, b1, nx, ny, nz, g.nb[0], g.st[0], g.ngap, g.nw, g.bw);
  MB2_LAUNCH_CHECK();
  wand_axis_kernel<<<grid, 256, 0, s>>>(b1, b2, g.nb[0], ny, nz, g.nb[1], g.st[1], g.ngap, g.nw);
  MB2_LAUNCH_CHECK();
  wand_axis_kernel<<<grid, 256, 0, s>>>(b2, b3, (long long)g.nb[0] * g.nb[1], nz, 1, g.nb[2],
                                        g.st[2], g.ngap, g.nw);
  MB2_LAUNCH_CHECK();
  *wand = b3;
  return MIRORR_OK;
}

const unsigned int *ncc_timeout_flag(const BmWork &w) {
  return w.ncc_ctl.ptr ? w.ncc_ctl.as<unsigned int>() + 5 : nullptr;
}

mirorr_status ncc_give_up_flag(BmWork &w, cudaStream_t s, unsigned int **flag) {
  const void *before = w.ncc_ctl.ptr;
  MB2_TRY(w.ncc_ctl.ensure(sizeof(unsigned int) * 8));
  if (w.ncc_ctl.ptr != before)
    MB2_CUDA_TRY(cudaMemsetAsync(w.ncc_ctl.ptr, 0, sizeof(unsigned int) * 8, s));
  *flag = w.ncc_ctl.as<unsigned int>() + 5;
  return MIRORR_OK;
}

mirorr_status ncc_take_timeout(BmWork &w, cudaStream_t s, bool *timed_out) {
  *timed_out = false;
  if (!w.ncc_ctl.ptr) return MIRORR_OK;
  unsigned int f = 0;
  unsigned int *flag = w.ncc_ctl.as<unsigned int>() + 5;
  MB2_CUDA_TRY(cudaMemcpyAsync(&f, flag, sizeof(f), cudaMemcpyDeviceToHost, s));
  MB2_CUDA_TRY(cudaStreamSynchronize(s));
  if (f) {
    MB2_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(f), s));
    *timed_out = true;
  }
  return MIRORR_OK;
}

}  // namespace mb2
