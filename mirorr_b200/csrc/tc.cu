// tc.cu -- the 16-bit storage search (BF16 or FP16 volumes) for sm_100a: the
// block-vs-window cross term of the NCC search on the tensor cores
// (tcgen05.mma, FP32 accumulation in tensor memory), the rest on the CUDA
// cores in FP32 (the box statistics from exact FP64 sums).
//
// Semantics are those of the reference matcher (itkBlockMatcher.txx:46-101,
// 631-848; see ncc.cu): for each block and each candidate of its clipped
// +-R window, mu_x, mu_y = means over all BW^3 voxels, m = base mask != 0 &&
// search mask != 0, Sxy = sum m (x - mu_x)(y - mu_y), Sxx, Syy likewise,
// score = Sxy^2 / Sxx / Syy or -2 when Sxx <= 0 or Syy <= 0; best and second
// as the sequential strict update in raster order starting from -3 (in
// parallel: best = the maximum, ties to the first candidate in raster order;
// second = the largest of the rest).  Here every sum is FP32 over the 16-bit
// stored values, so scores differ from the FP64 reference by rounding only.
//
// Compensated cross term.  The base block is centred in FP32 (x~ = x - mu_x)
// and split into two 16-bit parts, x~ = hi + lo + O(2^-16 |x~|), hi = T(x~),
// lo = T(x~ - hi); the window values y are the stored 16-bit values
// themselves, exact in the operands.  The tensor cores sum x~' y
// (x~' = hi + lo) in FP32; Sxy = sum x~' y - mu_y sum x~' removes the window
// mean afterwards (sum x~' is about 0, so nothing large cancels).  Sxx is an
// FP32 two-pass sum; the box statistics (mu_y, Syy) come from exact FP64 sums
// of the 16-bit window values.
//
// Tensor formulation (block width 4, window W <= 8, block gap 1).  A tile is
// up to 8 consecutive blocks of one row of the block grid (same by, bz).  With
// k the x offset in the tile's window (32 wide), for each base row (vz, vy):
//   A[(blk, s, split), k] = part_split(x~_blk)(k - G blk - s, vy, vz)   (M = 128)
//   B[(dz, py), k]        = window(k, py + vy, dz + vz)                 (N = 64)
// so D[(blk, s, split), (dz, py)] = sum over (vz, vy, k) of A B is the split
// part of the cross term of block blk at candidate (x shift s, y shift py,
// z shift dz).  A is a banded (Toeplitz) matrix the CUDA cores write into
// shared memory (each row's band only: the zeros around it are written once
// per launch and never touched again); B is the window itself, brought into
// shared memory by one TMA tensor copy of the search image in an x-chunked
// copy ([x / 8][z][y][x % 8], 16-byte rows), so that every (vz, vy, k-step)
// operand is a plain shared-memory descriptor into that one box (no im2col).
// 32 MMAs of 128 x 64 x 16 per tile, accumulating in tensor memory.  The
// epilogue reads D from tensor memory, adds the two split rows, forms the
// scores and reduces the top two per block.
//
// Every stage takes an array of matcher calls (grid.y or, for the tensor
// search, a flat tile numbering over the calls), so one launch serves one
// call or the calls of many image pairs at once.
//
// Blocks that do not fit the tensor form -- base block partly or wholly
// outside its mask, a window candidate whose footprint leaves the search
// mask, Sxx = 0 -- go to ncc_fb16_kernel, which evaluates the masked sums
// directly in FP32 (one CTA per block).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cfloat>
#include <mutex>

#include "kernels.cuh"

namespace mb2 {

namespace {

template <typename T> struct S16;
template <> struct S16<__nv_bfloat16> {
  static __device__ __forceinline__ float f(__nv_bfloat16 v) { return __bfloat162float(v); }
  static __device__ __forceinline__ __nv_bfloat16 t(float v) { return __float2bfloat16_rn(v); }
  static __device__ __forceinline__ uint32_t bits(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }
  static constexpr uint32_t kFmt = 1;  // tcgen05 instruction-descriptor operand format
};
template <> struct S16<__half> {
  static __device__ __forceinline__ float f(__half v) { return __half2float(v); }
  static __device__ __forceinline__ __half t(float v) { return __float2half_rn(v); }
  static __device__ __forceinline__ uint32_t bits(__half v) { return __half_as_ushort(v); }
  static constexpr uint32_t kFmt = 0;
};

constexpr int kBW = 4;          // block width of the tensor form
constexpr int kB = 64;          // voxels per block
constexpr int kTileBlocks = 8;  // blocks per tile (M = 8 blocks x 8 shifts x 2 parts)
constexpr int kXC = 4;          // 8-wide x chunks of the window box (32 x values)
constexpr int kSlots = 11;      // window rows per plane in the box (8 + BW - 1)
constexpr int kPlanes = 11;     // window planes in the box (8 + BW - 1)
constexpr int kBoxBytes = kXC * kPlanes * kSlots * 16;
constexpr uint32_t kSBO = kSlots * 16;          // next plane (next 8 rows of N)
constexpr uint32_t kLBO = kPlanes * kSlots * 16; // next x chunk (next 8 of K)
constexpr int kAStepBytes = 128 * 16 * 2;  // one 128 x 16 A operand: [k chunk][row group][8 rows][16 B]
constexpr int kAChunkSteps = 8;            // the (vy, k-step) operands of one vz
constexpr int kAChunkBytes = kAChunkSteps * kAStepBytes;
constexpr uint32_t kALBO = 16 * 128;       // next k chunk of A
constexpr uint32_t kASBO = 128;            // next 8 rows of A
constexpr int kTmemCols = 128;  // D: two accumulators of 64 FP32 columns (tiles alternate)



using Args16 = Match16Call;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory operand descriptor, no swizzle, K-major (canonical 8-row x
// 16-byte core matrices): start, leading (next K chunk) and stride (next 8
// rows) byte offsets, descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Waits for the phase of parity `parity` of the barrier to complete.  Each
// try_wait suspends the thread until the phase completes or about 20 us pass
// (no polling loop spends issue slots); after `limit` such waits (about
// limit x 20 us) the wait gives up and returns false.
constexpr int kWaitSuspendNs = 20000;
constexpr int kWaitLimit = 50000;  // about one second
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int limit = kWaitLimit) {
  for (int i = 0; i < limit; ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kWaitSuspendNs)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const void *map, int c0, int c1, int c2,
                                            int c3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
      " [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// Running best / second over a multiset of (score, raster index): best is
// the largest score, ties to the smallest index; second the largest of the
// rest.  Equal to the reference's sequential strict update in raster order.
struct Top2 {
  float b1, b2;
  long long i1;
};
__device__ __forceinline__ void top2_add(Top2 &t, float s, long long i) {
  if (s > t.b1 || (s == t.b1 && i < t.i1)) {
    t.b2 = t.b1;
    t.b1 = s;
    t.i1 = i;
  } else {
    t.b2 = fmaxf(t.b2, s);
  }
}
__device__ __forceinline__ void top2_merge(Top2 &t, const Top2 &u) {
  if (u.b1 > t.b1 || (u.b1 == t.b1 && u.i1 < t.i1)) {
    t.b2 = fmaxf(t.b1, fmaxf(t.b2, u.b2));
    t.b1 = u.b1;
    t.i1 = u.i1;
  } else {
    t.b2 = fmaxf(t.b2, fmaxf(u.b1, u.b2));
  }
}
__device__ __forceinline__ Top2 top2_shfl_xor(const Top2 &t, int m) {
  Top2 u;
  u.b1 = __shfl_xor_sync(0xffffffffu, t.b1, m);
  u.b2 = __shfl_xor_sync(0xffffffffu, t.b2, m);
  u.i1 = __shfl_xor_sync(0xffffffffu, t.i1, m);
  return u;
}

__device__ __forceinline__ void write_out(const Args16 &a, long long b, float best, float second,
                                          long long match, uint8_t status) {
  a.best[b] = best;
  a.second[b] = second;
  a.match[b] = (int32_t)match;
  a.status[b] = status;
}

// Clipped candidate range of one axis for block gap 1 (itkBlockMatcher.txx:744-756).
__device__ __forceinline__ void cand_range(int o, int S, int W, int BW, int &lo, int &hi) {
  lo = o - W / 2;
  hi = lo + W - 1;
  if (lo < 0) lo = 0;
  if (hi > S - BW) hi = S - BW;
}

// ---------------------------------------------------------------------------
// Box statistics of the 16-bit search image: per candidate origin p, the mean
// of the BW^3 footprint (every voxel) and Syy = sum (y - mean)^2, from the
// footprint's sum and sum of squares in FP64.  Both sums of 16-bit values are
// exact in FP64 (a square has at most 22 significant bits), and so is
// B^3 sum y^2 - (sum y)^2 (B^3 = BW^3 voxels): Syy is that over B^3, rounded
// once, and 0 exactly when the footprint is constant.  The sign bit of Syy
// is set when a search-mask voxel of the footprint is 0.
//
// Separable: a CTA of 32 x 8 threads owns 32 x 8 output columns and walks
// 16 output planes; per input plane it stages the (32 + BW - 1) x (8 + BW - 1)
// halo (values and mask) in shared memory, sums each row's BW-wide runs
// along x (FP64), then each thread sums BW of those along y and keeps the
// last BW planes' sums in registers for the z sum.  grid.y = call; grid.x
// strides over the tiles.
// ---------------------------------------------------------------------------
constexpr int kBsX = 32, kBsY = 8, kBsZ = 16;
__device__ __forceinline__ long long stats_tiles(const Args16 &a, int BW, int &tx, int &ty) {
  const int vx = a.nx - BW + 1, vy = a.ny - BW + 1, vz = a.nz - BW + 1;
  if (vx <= 0 || vy <= 0 || vz <= 0) return 0;
  tx = (vx + kBsX - 1) / kBsX;
  ty = (vy + kBsY - 1) / kBsY;
  return (long long)tx * ty * ((vz + kBsZ - 1) / kBsZ);
}

template <typename T, int BW>
__global__ void __launch_bounds__(256) box_stats16_kernel(const Args16 *calls) {
  constexpr int HX = kBsX + BW - 1, HY = kBsY + BW - 1;  // halo (35 x 11 for BW 4)
  constexpr int NB = BW * BW * BW;
  __shared__ float s_v[HY][HX + 1];
  __shared__ uint8_t s_m[HY][HX + 1];
  __shared__ double s_sx[HY][kBsX], s_sq[HY][kBsX];
  __shared__ uint8_t s_mx[HY][kBsX];
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  int ntx = 0, nty = 0;
  const long long ntiles = stats_tiles(a, BW, ntx, nty);
  const T *__restrict__ y = static_cast<const T *>(a.search);
  const uint8_t *__restrict__ ms = a.smask;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int tid = threadIdx.x, lx = tid & 31, ly = tid >> 5;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int x0 = (int)(t % ntx) * kBsX;
    const long long r = t / ntx;
    const int y0 = (int)(r % nty) * kBsY, z0 = (int)(r / nty) * kBsZ;
    // the previous BW - 1 planes' sums (sum, sum of squares, mask-AND)
    double zs[BW - 1], zq[BW - 1];
    unsigned zm[BW - 1];
#pragma unroll
    for (int k = 0; k < BW - 1; ++k) {
      zs[k] = zq[k] = 0.0;
      zm[k] = 0u;
    }
    const int zend = min(z0 + kBsZ + BW - 1, nz);
    for (int zi = z0; zi < zend; ++zi) {
      __syncthreads();  // the previous plane's x sums are read
      const long long plane = (long long)zi * ny;
      for (int i = tid; i < HY * HX; i += 256) {
        const int hy = i / HX, hx = i - hy * HX;
        const int gx = x0 + hx, gy = y0 + hy;
        float v = 0.f;
        uint8_t m = 0;
        if (gx < nx && gy < ny) {
          const long long q = (plane + gy) * nx + gx;
          v = S16<T>::f(y[q]);
          m = ms[q] != 0 ? 1 : 0;
        }
        s_v[hy][hx] = v;
        s_m[hy][hx] = m;
      }
      __syncthreads();
      for (int i = tid; i < HY * kBsX; i += 256) {
        const int hy = i >> 5, hx = i & 31;
        double sx = 0.0, sq = 0.0;
        unsigned mk = 1;
#pragma unroll
        for (int k = 0; k < BW; ++k) {
          const double v = (double)s_v[hy][hx + k];
          sx += v;
          sq = fma(v, v, sq);
          mk &= s_m[hy][hx + k];
        }
        s_sx[hy][hx] = sx;
        s_sq[hy][hx] = sq;
        s_mx[hy][hx] = (uint8_t)mk;
      }
      __syncthreads();
      double sy = 0.0, qy = 0.0;
      unsigned my = 1;
#pragma unroll
      for (int k = 0; k < BW; ++k) {
        sy += s_sx[ly + k][lx];
        qy += s_sq[ly + k][lx];
        my &= s_mx[ly + k][lx];
      }
      const int oz = zi - (BW - 1);
      const int ox = x0 + lx, oy = y0 + ly;
      if (oz >= z0 && ox <= nx - BW && oy <= ny - BW) {
        double S = sy, Q = qy;
        unsigned inm = my;
#pragma unroll
        for (int k = 0; k < BW - 1; ++k) {
          S += zs[k];
          Q += zq[k];
          inm &= zm[k];
        }
        // NB Q - S^2 is exact (both terms are), so Syy is rounded once
        const double syy = ((double)NB * Q - S * S) / (double)NB;
        const float f = (float)syy;
        a.stats[((long long)oz * ny + oy) * a.sp + ox] =
            make_float2((float)(S / (double)NB), inm ? f : -f - 0.0f);
      }
#pragma unroll
      for (int k = 0; k < BW - 2; ++k) {
        zs[k] = zs[k + 1];
        zq[k] = zq[k + 1];
        zm[k] = zm[k + 1];
      }
      zs[BW - 2] = sy;
      zq[BW - 2] = qy;
      zm[BW - 2] = my;
    }
  }
}

// ---------------------------------------------------------------------------
// Window-AND per block, separable (x over the rows, then y, then z at block
// resolution): 1 when every voxel of the block's clipped window box (the
// union of its candidates' footprints) is inside the search mask.
// ---------------------------------------------------------------------------
__global__ void wand_x16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const int R = a.W / 2;
  const long long n = (long long)a.nbx * a.ny * a.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(i % a.nbx);
    const long long yz = i / a.nbx;
    const int ox = a.stx + bx * a.G;
    int lo = ox - R, hi = ox + R;
    if (lo < 0) lo = 0;
    if (hi > a.nx - a.bw) hi = a.nx - a.bw;
    unsigned v = 1;
    const uint8_t *row = a.smask + yz * a.nx;
    for (int x = lo; x <= hi + a.bw - 1; ++x) v &= row[x] != 0 ? 1u : 0u;
    a.wand[i] = (uint8_t)v;
  }
}
__global__ void wand_y16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const int R = a.W / 2;
  const uint8_t *in = a.wand;
  uint8_t *out = a.wand + (long long)a.nbx * a.ny * a.nz;
  const long long n = (long long)a.nbx * a.nby * a.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(i % a.nbx);
    const long long r = i / a.nbx;
    const int by = (int)(r % a.nby), z = (int)(r / a.nby);
    const int oy = a.sty + by * a.G;
    int lo = oy - R, hi = oy + R;
    if (lo < 0) lo = 0;
    if (hi > a.ny - a.bw) hi = a.ny - a.bw;
    unsigned v = 1;
    for (int y = lo; y <= hi + a.bw - 1; ++y) v &= in[((long long)z * a.ny + y) * a.nbx + bx];
    out[i] = (uint8_t)v;
  }
}
__global__ void wand_z16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const int R = a.W / 2;
  const uint8_t *in = a.wand + (long long)a.nbx * a.ny * a.nz;
  uint8_t *out = a.wand + (long long)a.nbx * a.ny * a.nz + (long long)a.nbx * a.nby * a.nz;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < a.nblocks;
       b += (long long)gridDim.x * blockDim.x) {
    const long long bxy = b % ((long long)a.nbx * a.nby);
    const int bz = (int)(b / ((long long)a.nbx * a.nby));
    const int oz = a.stz + bz * a.G;
    int lo = oz - R, hi = oz + R;
    if (lo < 0) lo = 0;
    if (hi > a.nz - a.bw) hi = a.nz - a.bw;
    unsigned v = 1;
    for (int z = lo; z <= hi + a.bw - 1; ++z) v &= in[(long long)z * a.nbx * a.nby + bxy];
    out[b] = (uint8_t)v;
  }
}
__device__ __forceinline__ const uint8_t *wand_of(const Args16 &a) {
  return a.wand + (long long)a.nbx * a.ny * a.nz + (long long)a.nbx * a.nby * a.nz;
}

// ---------------------------------------------------------------------------
// Base-block preparation, 16 lanes per block (lane r = vz * 4 + vy holds base
// row r): the FP32 mean, the masked sums of x~ and x~^2, the base-mask mode
// and the two 16-bit parts of x~ (packed per (part, vz, vy) as two 32-bit
// words).  Sums over the block are half-warp shuffle trees.  grid.y = call.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float half_sum(float v) {
#pragma unroll
  for (int o = 8; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__global__ void __launch_bounds__(256) prep16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const T *__restrict__ x = static_cast<const T *>(a.base);
  const uint8_t *__restrict__ mb = a.bmask;
  const int nx = a.nx, ny = a.ny;
  const int r = threadIdx.x & 15;
  const unsigned half_mask = (threadIdx.x & 16) ? 0xFFFF0000u : 0x0000FFFFu;
  // every lane of a warp runs the same number of iterations (the half-warp
  // shuffles need both halves), blocks past the end idle
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long niter = (a.nblocks * 16 + nthreads - 1) / nthreads;
  for (long long it = 0; it < niter; ++it) {
    const long long b = (it * nthreads + blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 4;
    const bool live = b < a.nblocks;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    unsigned mbits = 0;
    if (live) {
      int bx, by, bz;
      split3(b, a.nbx, a.nby, bx, by, bz);
      const long long q = ((long long)(a.stz + bz * a.G + (r >> 2)) * ny + (a.sty + by * a.G + (r & 3))) * nx +
                          (a.stx + bx * a.G);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        v[i] = S16<T>::f(x[q + i]);
        mbits |= (mb[q + i] != 0 ? 1u : 0u) << i;
      }
    }
    const float mu = half_sum((v[0] + v[1]) + (v[2] + v[3])) * (1.0f / kB);
    float sxx = 0.f, sxt = 0.f, stc = 0.f;
    uint32_t hw[2] = {0u, 0u}, lw[2] = {0u, 0u};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float d = v[i] - mu;
      if ((mbits >> i) & 1u) {
        sxx = fmaf(d, d, sxx);
        sxt += d;
      }
      const T h = S16<T>::t(d);
      const T l = S16<T>::t(d - S16<T>::f(h));
      stc += S16<T>::f(h) + S16<T>::f(l);
      hw[i >> 1] |= S16<T>::bits(h) << (16 * (i & 1));
      lw[i >> 1] |= S16<T>::bits(l) << (16 * (i & 1));
    }
    sxx = half_sum(sxx);
    sxt = half_sum(sxt);
    stc = half_sum(stc);
    const unsigned full = __ballot_sync(0xffffffffu, mbits == 0xFu) & half_mask;
    const unsigned none = __ballot_sync(0xffffffffu, mbits == 0u) & half_mask;
    if (live) {
      uint32_t *xb = a.xs + b * 64;
      *reinterpret_cast<uint2 *>(xb + r * 2) = make_uint2(hw[0], hw[1]);
      *reinterpret_cast<uint2 *>(xb + 32 + r * 2) = make_uint2(lw[0], lw[1]);
      if (r == 0) {
        Prep16 pp;
        pp.mu = mu;
        pp.sxx = sxx;
        pp.sxt = sxt;
        pp.sxt_tc = stc;
        pp.mmode = full == half_mask ? 1 : (none == half_mask ? 2 : 0);
        // the block's route: culled by the selection (its record written
        // here), the tensor-core search (base block and every candidate
        // footprint inside the masks, Sxx > 0), else the direct search's list
        pp.route = 0;
        pp.pad[0] = pp.pad[1] = 0;
        if (a.selected && !a.selected[b]) {
          int bx, by, bz;
          split3(b, a.nbx, a.nby, bx, by, bz);
          write_out(a, b, -3.f, -3.f,
                    ((long long)(a.stz + bz * a.G) * ny + (a.sty + by * a.G)) * nx + (a.stx + bx * a.G), 0);
        } else if (a.tensor && pp.mmode == 1 && wand_of(a)[b] && sxx > 0.f) {
          pp.route = 1;
        } else {
          const unsigned int k = atomicAdd(&a.ctl[1], 1u);
          a.fb_list[k] = (int)b;
        }
        a.prep[b] = pp;
      }
    }
  }
}

// Base-block preparation for other block widths (no tensor form): one warp
// per block, lane l < BW^2 holds base row (vz, vy) = (l / BW, l % BW); the
// FP32 mean, the masked sums of x~ and x~^2, the base-mask mode and the
// block's route (culled, or the direct search's list).  grid.y = call.
template <typename T, int BW>
__global__ void __launch_bounds__(256) prep16w_kernel(const Args16 *calls) {
  static_assert(BW * BW <= 32, "one warp per block");
  constexpr int NB = BW * BW * BW;
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const T *__restrict__ x = static_cast<const T *>(a.base);
  const uint8_t *__restrict__ mb = a.bmask;
  const int nx = a.nx, ny = a.ny;
  const int lane = threadIdx.x & 31;
  const bool row = lane < BW * BW;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long b = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); b < a.nblocks;
       b += nwarps) {
    int bx, by, bz;
    split3(b, a.nbx, a.nby, bx, by, bz);
    const int ox = a.stx + bx * a.G, oy = a.sty + by * a.G, oz = a.stz + bz * a.G;
    float v[BW];
    unsigned mbits = 0;
    float sum = 0.f;
    if (row) {
      const long long q = ((long long)(oz + lane / BW) * ny + (oy + lane % BW)) * nx + ox;
#pragma unroll
      for (int i = 0; i < BW; ++i) {
        v[i] = S16<T>::f(x[q + i]);
        mbits |= (mb[q + i] != 0 ? 1u : 0u) << i;
        sum += v[i];
      }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const float mu = sum * (1.0f / NB);
    float sxx = 0.f, sxt = 0.f;
    if (row) {
#pragma unroll
      for (int i = 0; i < BW; ++i) {
        const float d = v[i] - mu;
        if ((mbits >> i) & 1u) {
          sxx = fmaf(d, d, sxx);
          sxt += d;
        }
      }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      sxx += __shfl_xor_sync(0xffffffffu, sxx, o);
      sxt += __shfl_xor_sync(0xffffffffu, sxt, o);
    }
    constexpr unsigned rows_mask = (BW * BW == 32) ? 0xffffffffu : ((1u << (BW * BW)) - 1u);
    const unsigned full = __ballot_sync(0xffffffffu, row && mbits == (1u << BW) - 1u) & rows_mask;
    const unsigned none = __ballot_sync(0xffffffffu, row && mbits == 0u) & rows_mask;
    if (lane == 0) {
      Prep16 pp;
      pp.mu = mu;
      pp.sxx = sxx;
      pp.sxt = sxt;
      pp.sxt_tc = 0.f;
      pp.mmode = full == rows_mask ? 1 : (none == rows_mask ? 2 : 0);
      pp.route = 0;
      pp.pad[0] = pp.pad[1] = 0;
      if (a.selected && !a.selected[b]) {
        write_out(a, b, -3.f, -3.f, ((long long)oz * ny + oy) * nx + ox, 0);
      } else {
        const unsigned int k = atomicAdd(&a.ctl[1], 1u);
        a.fb_list[k] = (int)b;
      }
      a.prep[b] = pp;
    }
  }
}

// ---------------------------------------------------------------------------
// x-chunked copy of the search image for the window tensor copies:
// out[((xc * nz + z) * ny + y)] = 8 values search(x0 + 8 xc + i, y, z), zero
// outside the image.  x0 = (block grid x start) - R, so every tile's window
// starts on a chunk boundary.  grid.y = call.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void chunk16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active || !a.tensor) return;
  const T *__restrict__ in = static_cast<const T *>(a.search);
  const long long n = (long long)a.nxc * a.nz * a.ny;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(r % a.ny);
    const long long t = r / a.ny;
    const int z = (int)(t % a.nz);
    const int xc = (int)(t / a.nz);
    const long long row = ((long long)z * a.ny + y) * a.nx;
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint32_t lo = 0u, hi = 0u;
      const int xa = a.chunk_x0 + 8 * xc + 2 * k, xb2 = xa + 1;
      if (xa >= 0 && xa < a.nx) lo = S16<T>::bits(in[row + xa]);
      if (xb2 >= 0 && xb2 < a.nx) hi = S16<T>::bits(in[row + xb2]);
      w[k] = lo | (hi << 16);
    }
    a.chunked[r] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// The call of a tile in the launch's flat tile numbering (calls in order).
__device__ __forceinline__ int call_of_tile(const Args16 *calls, int ncalls, long long tile) {
  int lo = 0, hi = ncalls - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (calls[mid].tile0 <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Where tile `tile` lies: its call, first block column and block row.
struct TilePos {
  int ci, bx0, by, bz;
};
__device__ __forceinline__ TilePos tile_pos(const Args16 *calls, int ncalls, long long tile) {
  TilePos p;
  p.ci = call_of_tile(calls, ncalls, tile);
  const Args16 &a = calls[p.ci];
  const int lt = (int)(tile - a.tile0);  // tiles of one call < 2^31
  const int tx = a.tiles_x, nby = a.nby;
  const int r = lt / tx;
  p.bx0 = (lt - r * tx) * a.bpt;
  p.bz = r / nby;
  p.by = r - p.bz * nby;
  return p;
}

// Top two over a thread's or a block's candidates with a 32-bit raster key
// (tile-local: (dz * 8 + py) * 8 + x shift; raster order of the candidates
// of one block), same rule as Top2.
struct Top2k {
  float b1, b2;
  int k1;
};
__device__ __forceinline__ void top2k_merge(Top2k &t, const Top2k &u) {
  if (u.b1 > t.b1 || (u.b1 == t.b1 && u.k1 < t.k1)) {
    t.b2 = fmaxf(t.b1, fmaxf(t.b2, u.b2));
    t.b1 = u.b1;
    t.k1 = u.k1;
  } else {
    t.b2 = fmaxf(t.b2, fmaxf(u.b1, u.b2));
  }
}
__device__ __forceinline__ Top2k top2k_shfl_xor(const Top2k &t, int m) {
  Top2k u;
  u.b1 = __shfl_xor_sync(0xffffffffu, t.b1, m);
  u.b2 = __shfl_xor_sync(0xffffffffu, t.b2, m);
  u.k1 = __shfl_xor_sync(0xffffffffu, t.k1, m);
  return u;
}

// ---------------------------------------------------------------------------
// The tensor-core search: a warp-specialised persistent kernel, one CTA of 16
// warps per SM, the CTA's tiles taken round-robin (tile = CTA + k x grid).
//
//   warp 2 (loader): lanes 0-7 make the tile's block records (which blocks
//     take the tensor form; blocks that do not are listed for the direct
//     search, unselected ones written out); lane 0 brings into a ring of
//     kLdSlots the tile's window box and the box of the search statistics
//     (TMA tensor copies) and its blocks' 16-bit parts (one bulk copy);
//   warp 1, one thread (control): issues the tile's 32 MMAs into one of two
//     accumulators in tensor memory (64 FP32 columns each);
//   warps 4-7 (producers): thread m writes row m of A -- the bands of both
//     k-steps -- into a ring of kASlots buffers of one vz each (8 operands);
//   warps 8-15 (epilogue): warp 8 + 4 h + q reads lanes 32q.. and columns
//     32h.. of a finished accumulator, scores the candidates against the
//     staged statistics and reduces the top two per block; one thread per
//     block writes the block's record.
//
// Row m = (blk = m / 16, x shift s = (m / 2) % 8, part = m % 2) of A and D;
// column n = (dz = n / 8, py = n % 8).  Every hand-off is an mbarrier:
//   l_full[s]  loader (records + copies)     -> everyone    slot s ready
//   l_empty[s] control commit, producers,
//              epilogue (1 + 128 + 256)      -> loader      slot s read
//   a_full[s]  producers (128 arrivals)      -> control     A slot s written
//   a_empty[s] control (tcgen05.commit)      -> producers   its multiplies done
//   d_full[d]  control (commit)              -> epilogue    accumulator d done
//   d_empty[d] epilogue (256 arrivals)       -> control     accumulator d read
// Every wait is bounded; a wait that gives up sets the call's flag and the
// CTA's, each role leaves its loop, and the loader and the control thread let
// their copies and multiplies land (bounded) before tensor memory is
// released.
// ---------------------------------------------------------------------------
constexpr int kASlots = 4;     // A ring: one vz (8 operands, 32 KB) per slot
constexpr int kLdSlots = 3;    // load ring
constexpr int kWsThreads = 512;
constexpr int kStX = 32, kStY = 8, kStZ = 8;                 // statistics box (float2)
constexpr uint32_t kLdBox = 0;                                // window box (kBoxBytes)
constexpr uint32_t kLdStats = 8192;                           // statistics box
constexpr uint32_t kStatsBytes = kStX * kStY * kStZ * 8;      // 16 KB
constexpr uint32_t kLdXs = kLdStats + kStatsBytes;            // blocks' 16-bit parts
constexpr uint32_t kLdPrep = kLdXs + kTileBlocks * 256;       // blocks' records (Prep16)
constexpr uint32_t kLdSlotBytes = 27 * 1024;
static_assert(kLdPrep + kTileBlocks * sizeof(Prep16) <= kLdSlotBytes, "load slot layout");
static_assert(kBoxBytes <= kLdStats, "window box fits its place in the slot");

struct TcBars {
  uint64_t l_full[kLdSlots], l_empty[kLdSlots];
  uint64_t a_full[kASlots], a_empty[kASlots];
  uint64_t d_full[2], d_empty[2];
};

// Where one tile lies (shared memory, one per load slot); its blocks'
// records (Prep16) and 16-bit parts are copied into the slot.
struct TileRec {
  long long b0;                    // index of the tile's first block
  int nblk;                        // blocks of the tile in the grid
  int ci, bx0, oy, oz, xs0;        // call, first block column, window origin, statistics box x
};

size_t tc_ws_smem_bytes() {
  return (size_t)kASlots * kAChunkBytes + (size_t)kLdSlots * kLdSlotBytes + 1024;
}

// phase-parity wait on a use count: the k-th completion of a barrier (k = 0,
// 1, ...) has parity k & 1
__device__ __forceinline__ bool wait_use(uint64_t *bar, long long k) {
  return mbar_wait(bar, (unsigned)(k & 1));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const void *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <typename T, int W>
__global__ void __launch_bounds__(kWsThreads, 1)
    ncc_tc_kernel(const Args16 *calls, int ncalls, long long total_tiles) {
  static_assert(W >= 2 && W <= 8, "window of the tensor form");
  constexpr int R = W / 2;
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t *const sbase = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(dsm) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t *const sa = sbase;                              // A ring
  uint8_t *const sld = sbase + kASlots * kAChunkBytes;    // load ring
  __shared__ __align__(8) TcBars bars;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_fail;
  __shared__ int s_ep_ok;
  __shared__ TileRec s_rec[kLdSlots];
  __shared__ Top2k s_part[2][kTileBlocks];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < kLdSlots; ++i) {
      mbar_init(&bars.l_full[i], 1);
      mbar_init(&bars.l_empty[i], 1 + 128 + 256);
    }
    for (int i = 0; i < kASlots; ++i) {
      mbar_init(&bars.a_full[i], 128);
      mbar_init(&bars.a_empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&bars.d_full[i], 1);
      mbar_init(&bars.d_empty[i], 256);
    }
    s_fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // A starts as zeros; each row later rewrites only the words of its band
  for (int i = tid; i < kASlots * kAChunkBytes / 16; i += kWsThreads)
    reinterpret_cast<uint4 *>(sa)[i] = make_uint4(0u, 0u, 0u, 0u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const long long first = blockIdx.x, step = gridDim.x;
  const long long ntile = first < total_tiles ? (total_tiles - first + step - 1) / step : 0;

  if (warp == 2) {
    // ======================= loader: records and copies ======================
    long long j = 0;
    int fail_ci = 0, map_call = -1, cur = -1;
    long long call_t0 = 0, call_end = -1;
    bool ok = true;
    for (; j < ntile; ++j) {
      const int ls = (int)(j % kLdSlots);
      int wok = 1;
      if (lane == 0 && j >= kLdSlots) wok = wait_use(&bars.l_empty[ls], j / kLdSlots - 1) && !s_fail;
      wok = __shfl_sync(0xffffffffu, wok, 0);
      if (!wok) {
        ok = false;
        break;
      }
      const long long tile = first + j * step;
      if (lane == 0) {
        // the tile's call and place, from the cached call when it is the same
        if (tile >= call_end) {
          cur = tile_pos(calls, ncalls, tile).ci;
          const Args16 &c = calls[cur];
          call_t0 = c.tile0;
          call_end = c.tile0 + c.ntiles;
        }
        const Args16 &a = calls[cur];
        fail_ci = cur;
        const int lt = (int)(tile - call_t0);
        const int tx = a.tiles_x, nby = a.nby;
        const int rr = lt / tx;
        const int bx0 = (lt - rr * tx) * a.bpt, bz = rr / nby, by = rr - bz * nby;
        TileRec &r = s_rec[ls];
        const int oy = a.sty + by * a.G, oz = a.stz + bz * a.G;
        const int x0 = a.stx + bx0 * a.G - R;  // the tile's first candidate x
        r.b0 = ((long long)bz * nby + by) * a.nbx + bx0;
        r.nblk = min(a.bpt, a.nbx - bx0);
        r.ci = cur;
        r.bx0 = bx0;
        r.oy = oy;
        r.oz = oz;
        r.xs0 = (x0 & 1) ? x0 - 1 : x0;  // even (16-byte aligned copy), <= x0
        if (cur != map_call) {
          // the call's copy descriptors were written by the host before the
          // launch; order the tensor-map proxy after them
          map_call = cur;
          asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(
                           reinterpret_cast<uint64_t>(a.tmap[0]))
                       : "memory");
          asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(
                           reinterpret_cast<uint64_t>(a.tmap[1]))
                       : "memory");
        }
        uint8_t *const slot = sld + (size_t)ls * kLdSlotBytes;
        const unsigned nb = (unsigned)r.nblk;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                         smem_u32(&bars.l_full[ls])),
                     "r"((unsigned)kBoxBytes + kStatsBytes + nb * 256u + nb * (unsigned)sizeof(Prep16))
                     : "memory");
        tma_load_4d(slot + kLdBox, a.tmap[0], 0, oy - R, oz - R, (a.G * bx0) >> 3, &bars.l_full[ls]);
        tma_load_3d(slot + kLdStats, a.tmap[1], 2 * r.xs0, oy - R, oz - R, &bars.l_full[ls]);
        bulk_load(slot + kLdXs, a.xs + r.b0 * 64, nb * 256u, &bars.l_full[ls]);
        bulk_load(slot + kLdPrep, a.prep + r.b0, nb * (unsigned)sizeof(Prep16), &bars.l_full[ls]);
      }
      __syncwarp();
    }
    if (!ok && lane == 0) {
      atomicExch(&calls[fail_ci].ctl[2], 1u);
      s_fail = 1;
    }
    // copies still in flight land before the CTA ends (bounded): the last
    // request of each slot
    if (lane == 0)
      for (long long k = max(j - kLdSlots, 0LL); k < j; ++k) wait_use(&bars.l_full[k % kLdSlots], k / kLdSlots);
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // ===================== control: the multiplies ===========================
      constexpr uint32_t idesc = (1u << 4) | (S16<T>::kFmt << 7) | (S16<T>::kFmt << 10) |
                                 ((uint32_t)(64 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
      long long j = 0;
      bool ok = true;
      for (; j < ntile && ok; ++j) {
        const int ls = (int)(j % kLdSlots), dacc = (int)(j & 1);
        if (!wait_use(&bars.l_full[ls], j / kLdSlots) || s_fail) { ok = false; break; }
        if (j >= 2 && !wait_use(&bars.d_empty[dacc], (j - 2) / 2)) { ok = false; break; }
        tc_fence_after();
        const uint32_t wb = smem_u32(sld + (size_t)ls * kLdSlotBytes + kLdBox);
        const uint32_t dst = tmem + (uint32_t)dacc * 64u;
        for (int vz = 0; vz < 4 && ok; ++vz) {
          const long long g = j * 4 + vz;
          const int as = (int)(g % kASlots);
          if (!wait_use(&bars.a_full[as], g / kASlots)) { ok = false; break; }
          tc_fence_after();
          const uint32_t ab = smem_u32(sa) + (uint32_t)as * kAChunkBytes;
#pragma unroll
          for (int jj = 0; jj < kAChunkSteps; ++jj) {
            const int vy = jj >> 1, ks = jj & 1;
            const uint64_t ad = sdesc(ab + (uint32_t)jj * kAStepBytes, kALBO, kASBO);
            const uint64_t bd = sdesc(wb + (uint32_t)(2 * ks) * kLBO + (uint32_t)vz * kSBO +
                                          (uint32_t)vy * 16u,
                                      kLBO, kSBO);
            const int acc = (vz | jj) != 0;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dst),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                : "memory");
          }
          tc_commit(&bars.a_empty[as]);
        }
        if (!ok) break;
        tc_commit(&bars.l_empty[ls]);
        tc_commit(&bars.d_full[dacc]);
      }
      if (!ok) {
        const long long tile = first + (j < ntile ? j : ntile - 1) * step;
        atomicExch(&calls[call_of_tile(calls, ncalls, tile)].ctl[2], 1u);
        s_fail = 1;
        // every issued multiply finishes: a commit on tile j's accumulator
        // barrier tracks all of them (the epilogue sees s_fail)
        if (j < ntile) {
          tc_commit(&bars.d_full[j & 1]);
          wait_use(&bars.d_full[j & 1], j / 2);
        }
      } else if (j > 0) {
        wait_use(&bars.d_full[(j - 1) & 1], (j - 1) / 2);
      }
    }
    __syncwarp();  // the warp leaves the role converged
  } else if (warp >= 4 && warp < 8) {
    // ======================= producers: the A bands ==========================
    const int m = tid - 128;  // row of A
    const int blk = m >> 4, sft = (m >> 1) & 7, part = m & 1;
    const uint32_t row_off = (uint32_t)(m >> 3) * kASBO + (uint32_t)(m & 7) * 16u;
    int band_call = -1;
    uint32_t off[2][3] = {{0u, 0u, 0u}, {0u, 0u, 0u}};
    unsigned msk[2] = {0u, 0u};
    bool odd = false;
    for (long long j = 0; j < ntile; ++j) {
      const int ls = (int)(j % kLdSlots);
      if (s_fail || !wait_use(&bars.l_full[ls], j / kLdSlots)) {
        s_fail = 1;
        break;
      }
      const TileRec &r = s_rec[ls];
      if (r.ci != band_call) {
        band_call = r.ci;
        const int G = calls[r.ci].G;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int t0 = G * blk + sft - 16 * h;
          const bool band = t0 < 16 && t0 + 4 > 0;
          odd = t0 & 1;  // the same for both halves
          const int c0 = t0 >= 0 ? (t0 >> 1) : -((1 - t0) >> 1);  // floor(t0 / 2)
          msk[h] = 0u;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int c = c0 + k;
            const bool on = band && c >= 0 && c < 8 && (k < 2 || odd);
            off[h][k] = on ? (uint32_t)(h * kAStepBytes + (c >> 2) * kALBO + (c & 3) * 4) : 0u;
            msk[h] |= (on ? 1u : 0u) << k;
          }
        }
      }
      const bool live = blk < r.nblk;
      uint2 xw[16];
      {
        const uint2 *xr = reinterpret_cast<const uint2 *>(sld + (size_t)ls * kLdSlotBytes + kLdXs +
                                                          blk * 256 + part * 128);
#pragma unroll
        for (int q2 = 0; q2 < 16; ++q2) xw[q2] = live ? xr[q2] : make_uint2(0u, 0u);
      }
      mbar_arrive(&bars.l_empty[ls]);  // the slot's parts are in registers
      bool ok = true;
#pragma unroll
      for (int vz = 0; vz < 4; ++vz) {
        const long long g = j * 4 + vz;
        const int as = (int)(g % kASlots);
        if (g >= kASlots && !wait_use(&bars.a_empty[as], g / kASlots - 1)) {
          ok = false;
          break;
        }
        uint8_t *const cb = sa + (size_t)as * kAChunkBytes + row_off;
#pragma unroll
        for (int vy = 0; vy < 4; ++vy) {
          const uint2 w2 = xw[vz * 4 + vy];
          uint32_t wv[3];
          if (odd) {
            wv[0] = w2.x << 16;
            wv[1] = __byte_perm(w2.x, w2.y, 0x5432);
            wv[2] = w2.y >> 16;
          } else {
            wv[0] = w2.x;
            wv[1] = w2.y;
            wv[2] = 0u;
          }
          uint8_t *const stp = cb + (size_t)(2 * vy) * kAStepBytes;
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int k = 0; k < 3; ++k)
              if ((msk[h] >> k) & 1u) *reinterpret_cast<uint32_t *>(stp + off[h][k]) = wv[k];
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive(&bars.a_full[as]);
      }
      if (!ok) {
        s_fail = 1;
        break;
      }
    }
    __syncwarp();
  } else if (warp >= 8) {
    // ======================= epilogue: scores and top two ====================
    const int et = tid - 256;  // 0..255
    const int q = warp & 3, half = (warp - 8) >> 2;
    const int m = 32 * q + lane;
    const int blk = m >> 4, sft = (m >> 1) & 7, part = m & 1;
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * q) << 16);
    const bool finisher = half == 0 && (lane & 15) == 0;
    const int dz0 = 4 * half + 2 * part;
    int cnt_call = -1;
    unsigned int cnt_blocks = 0;
    unsigned long long cnt_cands = 0;
    for (long long j = 0; j < ntile; ++j) {
      const int ls = (int)(j % kLdSlots), dacc = (int)(j & 1);
      // the slot and the accumulator: one thread waits, the epilogue warps agree
      if (et == 0)
        s_ep_ok = wait_use(&bars.l_full[ls], j / kLdSlots) && wait_use(&bars.d_full[dacc], j / 2) &&
                  !s_fail;
      __syncwarp();
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      if (!s_ep_ok) {
        if (et == 0) s_fail = 1;
        break;
      }
      tc_fence_after();
      float v[16];
      const uint32_t dcol = lane_addr + (uint32_t)dacc * 64u + (uint32_t)(32 * half);
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        uint32_t d[16];
        tmem_ld16(dcol + 16u * hh, d);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const float o = __shfl_xor_sync(0xffffffffu, __uint_as_float(d[jj]), 1);
          if (part == hh) v[jj] = __uint_as_float(d[jj]) + o;
        }
      }
      tc_fence_before();
      mbar_arrive(&bars.d_empty[dacc]);
      const TileRec &r = s_rec[ls];
      const Prep16 *const pr = reinterpret_cast<const Prep16 *>(sld + (size_t)ls * kLdSlotBytes + kLdPrep);
      const Args16 &a = calls[r.ci];
      const int nx = a.nx, ny = a.ny, nz = a.nz;
      const int oy = r.oy, oz = r.oz;
      const int ox = a.stx + (r.bx0 + blk) * a.G;
      const bool elig = blk < r.nblk && pr[blk].route == 1;
      // this thread's candidates: x shift sft, planes dz0 (jj < 8) and dz0 + 1
      // (jj >= 8), rows py = jj % 8; jj order is their raster order
      Top2k t2;
      t2.b1 = -3.f;
      t2.b2 = -3.f;
      t2.k1 = 0x7fffffff;
      int xlo, xhi, ylo, yhi, zlo, zhi;
      cand_range(ox, nx, W, kBW, xlo, xhi);
      cand_range(oy, ny, W, kBW, ylo, yhi);
      cand_range(oz, nz, W, kBW, zlo, zhi);
      const int cx = ox - R + sft;
      if (elig && sft < W && cx >= xlo && cx <= xhi) {
        // valid rows py in [pylo, pyhi], planes dz0 + h valid when zok[h];
        // the statistics box holds every candidate of the tile (zeros where
        // it leaves the volume), invalid ones are scored -FLT_MAX
        const int pylo = max(ylo - (oy - R), 0), pyhi = min(yhi - (oy - R), W - 1);
        const int cz0 = oz - R + dz0;
        const bool zok0 = dz0 < W && cz0 >= zlo && cz0 <= zhi;
        const bool zok1 = dz0 + 1 < W && cz0 + 1 >= zlo && cz0 + 1 <= zhi;
        const unsigned rows = ((2u << pyhi) - 1u) & ~((1u << pylo) - 1u);
        const unsigned vmask = (zok0 ? rows : 0u) | (zok1 ? rows << 8 : 0u);
        const float2 *sst = reinterpret_cast<const float2 *>(sld + (size_t)ls * kLdSlotBytes + kLdStats) +
                            (dz0 * kStY) * kStX + (cx - r.xs0);
        const float sxx = pr[blk].sxx, stc = pr[blk].sxt_tc;
        int kbest = -1;
        float b1 = -3.f, b2 = -3.f;
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const float2 st = sst[((jj >> 3) * kStY + (jj & 7)) * kStX];
          const float sxy = fmaf(-st.x, stc, v[jj]);
          float sc = st.y > 0.f ? __fdividef(sxy * sxy, sxx * st.y) : -2.f;
          sc = ((vmask >> jj) & 1u) ? sc : -FLT_MAX;
          const bool gt = sc > b1;
          b2 = gt ? b1 : fmaxf(b2, sc);
          b1 = gt ? sc : b1;
          kbest = gt ? jj : kbest;
        }
        if (kbest >= 0) {
          t2.b1 = b1;
          t2.b2 = b2;
          t2.k1 = ((dz0 + (kbest >> 3)) * 8 + (kbest & 7)) * 8 + sft;
        }
      }
      // reduce over the 16 lanes of the block (8 shifts x 2 parts) ...
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) top2k_merge(t2, top2k_shfl_xor(t2, o));
      // ... then over the two halves of the candidate planes
      if (half == 1 && (lane & 15) == 0) s_part[j & 1][blk] = t2;
      __syncwarp();
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      if (finisher && elig) {
        top2k_merge(t2, s_part[j & 1][blk]);
        const int k = t2.k1;
        const long long idx =
            ((long long)(oz - R + (k >> 6)) * ny + (oy - R + ((k >> 3) & 7))) * nx + (ox - R + (k & 7));
        write_out(a, r.b0 + blk, t2.b1, t2.b2, idx, 1);
        if (r.ci != cnt_call) {
          if (cnt_call >= 0) {
            atomicAdd(&calls[cnt_call].ctl[0], cnt_blocks);
            if (calls[cnt_call].ncc_count) atomicAdd(calls[cnt_call].ncc_count, cnt_cands);
          }
          cnt_call = r.ci;
          cnt_blocks = 0;
          cnt_cands = 0;
        }
        ++cnt_blocks;
        cnt_cands += (unsigned long long)(xhi - xlo + 1) * (yhi - ylo + 1) * (zhi - zlo + 1);
      }
      __syncwarp();
      mbar_arrive(&bars.l_empty[ls]);  // the slot's records and statistics are read
    }
    if (finisher && cnt_call >= 0 && cnt_blocks) {
      atomicAdd(&calls[cnt_call].ctl[0], cnt_blocks);
      if (calls[cnt_call].ncc_count) atomicAdd(calls[cnt_call].ncc_count, cnt_cands);
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
}

// ---------------------------------------------------------------------------
// Direct FP32 search for the blocks the tensor form does not take (each
// call's fb_list; block width 5 takes every block here): one CTA per block.
// The window (at most 16^3 values) and the base block are staged in shared
// memory; window rows are 18 floats apart and planes 16 x 18 + 6, so the
// rows the threads of a warp read (11 strips per plane at window 11) start on
// distinct bank pairs and a row is read with 8-byte loads.  Thread t owns the x strip of candidates at
// (py, pz) = (t % ncy, t / ncy): per base row (vy, vz) it reads the window row
// once and updates all its candidates' cross terms from registers, in the
// raster order of the base block, so each candidate's sum is the one a
// per-candidate loop forms (windows of more than 128 strips deal them
// round-robin).  A candidate whose footprint lies inside the
// search mask with the base block inside its mask is scored from that cross
// term and the box statistics (Syy); any other candidate is re-summed with
// the masked sums of the reference formula.  grid.y = call.
// ---------------------------------------------------------------------------
template <typename T, int BW>
__global__ void __launch_bounds__(128, 8) ncc_fb16_kernel(const Args16 *calls) {
  constexpr int NT = 128;
  constexpr int NB = BW * BW * BW;
  constexpr int RS = 18;             // window row stride (floats)
  constexpr int PS = 16 * RS + 6;    // window plane stride (floats)
  constexpr int NCX = 16 - BW + 1;   // longest x strip (window extent <= 16)
  __shared__ float s_xt[NB], s_mb[NB];
  __shared__ __align__(16) float s_y[16 * PS];
  __shared__ uint8_t s_m[16 * PS];
  __shared__ Top2 s_red[NT / 32];
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const int tid = threadIdx.x;
  const T *base = static_cast<const T *>(a.base);
  const T *search = static_cast<const T *>(a.search);
  const unsigned int nlist = *(volatile unsigned int *)&a.ctl[1];
  for (unsigned int li = blockIdx.x; li < nlist; li += gridDim.x) {
    const long long b = a.fb_list[li];
    int bx, by, bz;
    split3(b, a.nbx, a.nby, bx, by, bz);
    const int ox = a.stx + bx * a.G, oy = a.sty + by * a.G, oz = a.stz + bz * a.G;
    int xlo, xhi, ylo, yhi, zlo, zhi;
    cand_range(ox, a.nx, a.W, BW, xlo, xhi);
    cand_range(oy, a.ny, a.W, BW, ylo, yhi);
    cand_range(oz, a.nz, a.W, BW, zlo, zhi);
    const int ncx = xhi - xlo + 1, ncy = yhi - ylo + 1, ncz = zhi - zlo + 1;
    const int ex = ncx + BW - 1, ey = ncy + BW - 1, ez = ncz + BW - 1;
    const Prep16 pp = a.prep[b];
    __syncthreads();
    for (int t = tid; t < NB; t += NT) {
      const int vx = t % BW, vy = (t / BW) % BW, vz = t / (BW * BW);
      const long long qq = ((long long)(oz + vz) * a.ny + (oy + vy)) * a.nx + (ox + vx);
      const float mv = a.bmask[qq] != 0 ? 1.f : 0.f;
      s_xt[t] = S16<T>::f(base[qq]) - pp.mu;
      s_mb[t] = mv;
    }
    {
      // a 16-lane group per window row (ex <= 16); the group's row (wy, wz)
      // advances by NT / 16 rows without a division
      const int wx = tid & 15;
      int wy = tid >> 4, wz = ncx > 0 && ncy > 0 && ncz > 0 ? 0 : ez;  // empty window: none
      while (wz < ez && wy >= ey) {
        wy -= ey;
        ++wz;
      }
      // four rows per pass, all of their loads issued before the stores
      while (wz < ez) {
        T yv[4];
        uint8_t mv[4];
        int so[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          so[j] = -1;
          if (wz < ez && wx < ex) {
            const long long qq = ((long long)(zlo + wz) * a.ny + (ylo + wy)) * a.nx + (xlo + wx);
            yv[j] = search[qq];
            mv[j] = a.smask[qq];
            so[j] = wz * PS + wy * RS + wx;
          }
          wy += NT / 16;
          while (wz < ez && wy >= ey) {
            wy -= ey;
            ++wz;
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (so[j] >= 0) {
            s_y[so[j]] = S16<T>::f(yv[j]);
            s_m[so[j]] = mv[j] != 0 ? 1 : 0;
          }
      }
    }
    __syncthreads();
    Top2 tp;
    tp.b1 = -3.f;
    tp.b2 = -3.f;
    tp.i1 = 0x7fffffffffffffffLL;
    const int nc = ncx * ncy * ncz;
    for (int strip = tid; strip < ncy * ncz; strip += NT) {
      const int py = strip % ncy, pz = strip / ncy;
      const int cy = ylo + py, cz = zlo + pz;
      // the strip's cross terms (base block inside its mask only)
      float acc[NCX];
#pragma unroll
      for (int px = 0; px < NCX; ++px) acc[px] = 0.f;
      if (pp.mmode == 1) {
        for (int vz = 0; vz < BW; ++vz)
#pragma unroll
          for (int vy = 0; vy < BW; ++vy) {
            // values past the window's extent only feed strip positions
            // px >= ncx, which are not scored
            const float2 *row = reinterpret_cast<const float2 *>(s_y + (pz + vz) * PS + (py + vy) * RS);
            float r[16];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const float2 q = row[k];
              r[2 * k] = q.x;
              r[2 * k + 1] = q.y;
            }
            float t[BW];
#pragma unroll
            for (int vx = 0; vx < BW; ++vx) t[vx] = s_xt[(vz * BW + vy) * BW + vx];
#pragma unroll
            for (int px = 0; px < NCX; ++px)
#pragma unroll
              for (int vx = 0; vx < BW; ++vx) acc[px] = fmaf(t[vx], r[px + vx], acc[px]);
          }
      }
#pragma unroll
      for (int px = 0; px < NCX; ++px) {
        if (px >= ncx) break;
        const int cx = xlo + px;
        const long long idx = ((long long)cz * a.ny + cy) * a.nx + cx;
        const float2 st = __ldg(a.stats + ((long long)cz * a.ny + cy) * a.sp + cx);
        const float muy = st.x;
        float sxy = 0.f, sxx = 0.f, syy = 0.f;
        if (pp.mmode == 1 && !signbit(st.y)) {
          // footprint and base block wholly inside their masks
          sxy = acc[px] - muy * pp.sxt;
          sxx = pp.sxx;
          syy = st.y;
        } else {
#pragma unroll 5
          for (int i = 0; i < NB; ++i) {
            const int vx = i % BW, vy = (i / BW) % BW, vz = i / (BW * BW);
            const int w = (pz + vz) * PS + (py + vy) * RS + px + vx;
            const float mk = s_mb[i] * (float)s_m[w];
            const float dy = s_y[w] - muy;
            const float xm = mk * s_xt[i];
            sxy = fmaf(xm, dy, sxy);
            sxx = fmaf(xm, s_xt[i], sxx);
            syy = fmaf(mk * dy, dy, syy);
          }
        }
        const float sc = (sxx <= 0.f || syy <= 0.f) ? -2.f : __fdividef(sxy * sxy, sxx * syy);
        top2_add(tp, sc, idx);
      }
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) top2_merge(tp, top2_shfl_xor(tp, o));
    if ((tid & 31) == 0) s_red[tid >> 5] = tp;
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < NT / 32; ++w) top2_merge(tp, s_red[w]);
      const long long orig = ((long long)oz * a.ny + oy) * a.nx + ox;
      if (nc > 0) write_out(a, b, tp.b1, tp.b2, tp.i1, 1);
      else write_out(a, b, -3.f, -3.f, orig, 1);
      if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)nc);
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  });
  return fn;
}


}  // namespace

// Derived per-call fields: the tensor form's tile layout and copy geometry.
void prepare16(const BmGeom &g, Match16Call &c) {
  c.nx = g.size[0]; c.ny = g.size[1]; c.nz = g.size[2];
  c.sp = (c.nx + 1) & ~1;
  c.nbx = g.nb[0]; c.nby = g.nb[1]; c.nbz = g.nb[2];
  c.stx = g.st[0]; c.sty = g.st[1]; c.stz = g.st[2];
  c.G = g.ngap;
  c.W = g.nw;
  c.bw = g.bw;
  c.nblocks = g.nblocks;
  // blocks per tile: the tile's bands fit the 32-wide box, and G bpt is a
  // multiple of 8 so every tile's window starts on a chunk of the copy
  c.bpt = 0;
  for (int b = kTileBlocks; b >= 1; --b)
    if (g.ngap * (b - 1) + g.nw + kBW - 1 <= 8 * kXC && (g.ngap * b) % 8 == 0) {
      c.bpt = b;
      break;
    }
  c.tensor = g.bw == kBW && g.bgap == 1 && (g.nw & 1) && g.nw <= 7 && g.nw >= 3 && c.bpt > 0 &&
             c.ny >= kSlots && c.nz >= kPlanes;
  c.tiles_x = c.tensor ? (g.nb[0] + c.bpt - 1) / c.bpt : 0;
  c.ntiles = (long long)c.tiles_x * g.nb[1] * g.nb[2];
  c.chunk_x0 = g.st[0] - g.nw / 2;
  c.nxc = c.tensor ? (g.ngap * c.bpt / 8) * (c.tiles_x - 1) + kXC : 0;
}

size_t match16_chunk_bytes(const Match16Call &c) {
  return c.tensor ? sizeof(uint4) * (size_t)c.nxc * c.nz * c.ny : 0;
}

long long match16_number_tiles(Match16Call *calls, int n) {
  long long tiles = 0;
  for (int i = 0; i < n; ++i) {
    calls[i].tile0 = tiles;
    if (calls[i].active && calls[i].tensor) tiles += calls[i].ntiles;
  }
  return tiles;
}

mirorr_status match16_prepare_copies(int dtype, Match16Call *calls, int n) {
  EncodeTiledFn enc = nullptr;
  for (int i = 0; i < n; ++i) {
    Match16Call &c = calls[i];
    memset(c.tmap, 0, sizeof(c.tmap));
    if (!c.active || !c.tensor) continue;
    if (!enc) {
      enc = encode_fn();
      if (!enc) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return MIRORR_ECUDA;
      }
    }
    CUtensorMap *m = reinterpret_cast<CUtensorMap *>(c.tmap[0]);
    {
      // the window box: [x / 8][z][y][x % 8] 16-bit values, box 8 x 11 x 11 x 4
      const cuuint64_t dims[4] = {8, (cuuint64_t)c.ny, (cuuint64_t)c.nz, (cuuint64_t)c.nxc};
      const cuuint64_t strides[3] = {16, (cuuint64_t)16 * c.ny, (cuuint64_t)16 * c.ny * c.nz};
      const cuuint32_t box[4] = {8, (cuuint32_t)kSlots, (cuuint32_t)kPlanes, (cuuint32_t)kXC};
      const cuuint32_t estr[4] = {1, 1, 1, 1};
      const CUresult r = enc(&m[0],
                             dtype == MIRORR_DTYPE_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                        : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                             4, c.chunked, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (window box) failed (%d)", (int)r);
        return MIRORR_ECUDA;
      }
    }
    {
      // the statistics box: float2 rows of pitch sp seen as pairs of float32,
      // box 32 positions x 8 rows x 8 planes
      const cuuint64_t dims[3] = {(cuuint64_t)2 * c.sp, (cuuint64_t)c.ny, (cuuint64_t)c.nz};
      const cuuint64_t strides[2] = {(cuuint64_t)8 * c.sp, (cuuint64_t)8 * c.sp * c.ny};
      const cuuint32_t box[3] = {(cuuint32_t)(2 * kStX), (cuuint32_t)kStY, (cuuint32_t)kStZ};
      const cuuint32_t estr[3] = {1, 1, 1};
      const CUresult r = enc(&m[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, c.stats, dims, strides, box,
                             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (statistics box) failed (%d)", (int)r);
        return MIRORR_ECUDA;
      }
    }
  }
  return MIRORR_OK;
}

size_t match16_stats_bytes(const Match16Call &c) {
  return sizeof(float2) * (size_t)c.sp * c.ny * c.nz;
}

size_t match16_wand_bytes(const Match16Call &c) {
  return (size_t)c.nbx * c.ny * c.nz + (size_t)c.nbx * c.nby * c.nz + (size_t)c.nblocks;
}

namespace {

template <typename T>
mirorr_status run16(int ncalls, Match16Call *host_calls, DevBuf &calls_dev, cudaStream_t s,
                    bool every_stage) {
  const int SM = sm_count();
  const long long tiles = match16_number_tiles(host_calls, ncalls);
  MB2_TRY(match16_prepare_copies(S16<T>::kFmt == 1 ? MIRORR_DTYPE_BF16 : MIRORR_DTYPE_F16, host_calls,
                                 ncalls));
  long long max_vox = 0, max_blocks = 0, max_chunks = 0;
  int W = 0, G = 0, BWc = 0;
  bool any_tensor = false;
  for (int i = 0; i < ncalls; ++i) {
    const Match16Call &c = host_calls[i];
    if (c.active) {
      if (BWc && BWc != c.bw) {
        set_error("the calls of one launch must share the block width");
        return MIRORR_EINVAL;
      }
      BWc = c.bw;
    }
    if (c.active && c.tensor) {
      any_tensor = true;
      if ((W && W != c.W) || (G && G != c.G)) {
        set_error("the calls of one launch must share the window and the block spacing");
        return MIRORR_EINVAL;
      }
      W = c.W;
      G = c.G;
    }
    if (!c.active) continue;
    max_vox = std::max(max_vox, (long long)c.nx * c.ny * c.nz);
    max_blocks = std::max(max_blocks, c.nblocks);
    max_chunks = std::max(max_chunks, (long long)c.nxc * c.nz * c.ny);
  }
  MB2_TRY(calls_dev.ensure(sizeof(Args16) * ncalls));
  MB2_CUDA_TRY(cudaMemcpyAsync(calls_dev.ptr, host_calls, sizeof(Args16) * ncalls,
                               cudaMemcpyHostToDevice, s));
  const Args16 *dc = calls_dev.as<Args16>();
  auto grid_for = [&](long long n) {
    long long b = (n + 255) / 256;
    if (b > (long long)SM * 4) b = (long long)SM * 4;
    return dim3((unsigned)(b < 1 ? 1 : b), (unsigned)ncalls);
  };
  {
    long long st_tiles = 0;
    for (int i = 0; i < ncalls; ++i) {
      const Match16Call &c = host_calls[i];
      if (!c.active) continue;
      const long long vx = c.nx - c.bw + 1, vy = c.ny - c.bw + 1, vz = c.nz - c.bw + 1;
      if (vx > 0 && vy > 0 && vz > 0)
        st_tiles = std::max(st_tiles, ((vx + kBsX - 1) / kBsX) * ((vy + kBsY - 1) / kBsY) *
                                          ((vz + kBsZ - 1) / kBsZ));
    }
    long long gx = std::min(st_tiles, (long long)SM * 8);
    if (gx < 1) gx = 1;
    if (BWc == 5) box_stats16_kernel<T, 5><<<dim3((unsigned)gx, (unsigned)ncalls), 256, 0, s>>>(dc);
    else box_stats16_kernel<T, 4><<<dim3((unsigned)gx, (unsigned)ncalls), 256, 0, s>>>(dc);
  }
  MB2_LAUNCH_CHECK();
  wand_x16_kernel<<<grid_for(max_vox / 2 + 1), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  wand_y16_kernel<<<grid_for(max_vox / 4 + 1), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  wand_z16_kernel<<<grid_for(max_blocks), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  if (BWc == 5) prep16w_kernel<T, 5><<<grid_for(max_blocks * 32), 256, 0, s>>>(dc);
  else prep16_kernel<T><<<grid_for(max_blocks * 16), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  if (any_tensor || every_stage) {
    chunk16_kernel<T><<<grid_for(max_chunks), 256, 0, s>>>(dc);
    MB2_LAUNCH_CHECK();
  }
  if (any_tensor || every_stage) {
    const size_t smem = tc_ws_smem_bytes();
    auto kern = (W == 7) ? ncc_tc_kernel<T, 7> : (W == 5) ? ncc_tc_kernel<T, 5>
                                                          : ncc_tc_kernel<T, 3>;
    MB2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    long long grid = tiles < (long long)SM ? tiles : (long long)SM;
    // with every stage launched (a graph of fixed shape), a launch without
    // tensor tiles is one CTA that finds no tile
    if (grid < 1 && every_stage) grid = 1;
    if (grid > 0) {
      kern<<<(unsigned)grid, kWsThreads, smem, s>>>(dc, ncalls, tiles);
      MB2_LAUNCH_CHECK();
    }
  }
  if (BWc == 5) ncc_fb16_kernel<T, 5><<<dim3((unsigned)SM * 8, (unsigned)ncalls), 128, 0, s>>>(dc);
  else ncc_fb16_kernel<T, 4><<<dim3((unsigned)SM * 8, (unsigned)ncalls), 128, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace

mirorr_status launch_match16_batch(int dtype, int ncalls, Match16Call *host_calls,
                                   DevBuf &calls_dev, cudaStream_t s, bool every_stage) {
  if (ncalls <= 0) return MIRORR_OK;
  if (dtype == MIRORR_DTYPE_BF16)
    return run16<__nv_bfloat16>(ncalls, host_calls, calls_dev, s, every_stage);
  if (dtype == MIRORR_DTYPE_F16) return run16<__half>(ncalls, host_calls, calls_dev, s, every_stage);
  set_error("storage type %d is not a 16-bit type", dtype);
  return MIRORR_EINVAL;
}

mirorr_status launch_match16(int dtype, const BmGeom &g, const void *base, const uint8_t *bmask,
                             const void *search, const uint8_t *smask, const uint8_t *selected,
                             const BmOut &out, Bm16Work &w, unsigned long long *ncc_count,
                             cudaStream_t s) {
  if (g.bw != 4 && g.bw != 5) {
    set_error("the 16-bit search supports block widths 4 and 5 (got %d)", g.bw);
    return MIRORR_EINVAL;
  }
  if (g.bgap != 1) {
    set_error("the 16-bit search supports block gap 1 (got %d)", g.bgap);
    return MIRORR_EINVAL;
  }
  if (g.nw + g.bw - 1 > 16) {
    set_error("the 16-bit search supports windows up to %d for block width %d (got %d)",
              17 - g.bw, g.bw, g.nw);
    return MIRORR_EINVAL;
  }
  Match16Call c;
  memset(&c, 0, sizeof(c));
  prepare16(g, c);
  MB2_TRY(w.stats.ensure(match16_stats_bytes(c)));
  MB2_TRY(w.wand.ensure(match16_wand_bytes(c)));
  MB2_TRY(w.prep.ensure(sizeof(Prep16) * g.nblocks));
  MB2_TRY(w.xs.ensure(sizeof(uint32_t) * 64 * g.nblocks));
  MB2_TRY(w.ctl.ensure(4 * sizeof(unsigned int)));
  MB2_TRY(w.fb_list.ensure(sizeof(int) * g.nblocks));
  if (c.tensor) MB2_TRY(w.chunked.ensure(match16_chunk_bytes(c)));
  MB2_CUDA_TRY(cudaMemsetAsync(w.ctl.ptr, 0, 4 * sizeof(unsigned int), s));
  c.base = base;
  c.bmask = bmask;
  c.search = search;
  c.smask = smask;
  c.selected = selected;
  c.stats = w.stats.as<float2>();
  c.wand = w.wand.as<uint8_t>();
  c.prep = w.prep.as<Prep16>();
  c.xs = w.xs.as<uint32_t>();
  c.chunked = w.chunked.as<uint4>();
  c.best = out.best;
  c.second = out.second;
  c.match = out.match;
  c.status = out.status;
  c.ncc_count = ncc_count;
  c.ctl = w.ctl.as<unsigned int>();
  c.fb_list = w.fb_list.as<int>();
  c.active = 1;
  return launch_match16_batch(dtype, 1, &c, w.calls, s);
}

size_t match16_prep_bytes() { return sizeof(Prep16); }

mirorr_status match16_take_timeout(Bm16Work &w, cudaStream_t s, bool *timed_out) {
  *timed_out = false;
  if (!w.ctl.ptr) return MIRORR_OK;
  unsigned int f = 0;
  unsigned int *flag = w.ctl.as<unsigned int>() + 2;
  MB2_CUDA_TRY(cudaMemcpyAsync(&f, flag, sizeof(f), cudaMemcpyDeviceToHost, s));
  MB2_CUDA_TRY(cudaStreamSynchronize(s));
  *timed_out = f != 0;
  return MIRORR_OK;
}

mirorr_status match16_counts(Bm16Work &w, cudaStream_t s, unsigned int out[2]) {
  out[0] = out[1] = 0;
  if (!w.ctl.ptr) return MIRORR_OK;
  MB2_CUDA_TRY(cudaMemcpyAsync(out, w.ctl.ptr, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  MB2_CUDA_TRY(cudaStreamSynchronize(s));
  return MIRORR_OK;
}

}  // namespace mb2
