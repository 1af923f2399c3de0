// tc.cu -- the 16-bit storage search (BF16 or FP16 volumes) for sm_100a: the
// block-vs-window cross term of the NCC search on the tensor cores
// (tcgen05.mma, FP32 accumulation in tensor memory), the rest on the CUDA
// cores in FP32.  No FP64 anywhere in this file.
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
// mean afterwards (sum x~' is about 0, so nothing large cancels).  Sxx and the
// box statistics (mu_y, Syy) are FP32 two-pass sums.
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
constexpr int kCtasPerSM = 3;              // resident CTAs per SM (their phases overlap)
constexpr uint32_t kALBO = 16 * 128;       // next k chunk of A
constexpr uint32_t kASBO = 128;            // next 8 rows of A
constexpr int kTmemCols = 64;   // D: 64 columns of FP32
constexpr int kThreads = 256;
constexpr int kMaxCalls = 128;  // tensor maps of one launch (kernel parameter space)



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

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            int c3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
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
__device__ __forceinline__ void cand_range(int o, int S, int W, int &lo, int &hi) {
  lo = o - W / 2;
  hi = lo + W - 1;
  if (lo < 0) lo = 0;
  if (hi > S - kBW) hi = S - kBW;
}

// ---------------------------------------------------------------------------
// Box statistics of the 16-bit search image: per candidate origin p, the mean
// of the BW^3 footprint (every voxel) and sum (y - mean)^2, FP32 two-pass;
// the sign bit of Syy is set when a search-mask voxel of the footprint is 0.
// One thread per 4 consecutive x positions (each footprint row of 7 values
// serves the 4).  grid.y = call.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) box_stats16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const T *__restrict__ y = static_cast<const T *>(a.search);
  const uint8_t *__restrict__ ms = a.smask;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  float2 *__restrict__ out = a.stats;
  constexpr int PX = 4, RL = PX + kBW - 1;
  const int ngx = (nx + PX - 1) / PX;
  const long long n = (long long)ngx * ny * nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    int gx, yy, z;
    split3(p, ngx, ny, gx, yy, z);
    const int x0 = gx * PX;
    const long long o = ((long long)z * ny + yy) * nx + x0;
    const bool rowok = yy <= ny - kBW && z <= nz - kBW;
    float sum[PX], ss[PX];
    unsigned allm = ~0u;
#pragma unroll
    for (int j = 0; j < PX; ++j) sum[j] = ss[j] = 0.f;
    if (rowok && x0 <= nx - kBW) {
#pragma unroll
      for (int vz = 0; vz < kBW; ++vz)
#pragma unroll
        for (int vy = 0; vy < kBW; ++vy) {
          const long long q = o + ((long long)vz * ny + vy) * nx;
          float v[RL];
          unsigned mb = 0u;
#pragma unroll
          for (int i = 0; i < RL; ++i) {
            const bool in = x0 + i < nx;
            v[i] = in ? S16<T>::f(y[q + i]) : 0.f;
            mb |= ((in && ms[q + i] != 0) ? 1u : 0u) << i;
          }
          allm &= mb;
#pragma unroll
          for (int vx = 0; vx < kBW; ++vx)
#pragma unroll
            for (int j = 0; j < PX; ++j) sum[j] += v[j + vx];
        }
      float mu[PX];
#pragma unroll
      for (int j = 0; j < PX; ++j) mu[j] = sum[j] * (1.0f / kB);
#pragma unroll
      for (int vz = 0; vz < kBW; ++vz)
#pragma unroll
        for (int vy = 0; vy < kBW; ++vy) {
          const long long q = o + ((long long)vz * ny + vy) * nx;
          float v[RL];
#pragma unroll
          for (int i = 0; i < RL; ++i) v[i] = (x0 + i < nx) ? S16<T>::f(y[q + i]) : 0.f;
#pragma unroll
          for (int vx = 0; vx < kBW; ++vx)
#pragma unroll
            for (int j = 0; j < PX; ++j) {
              const float d = v[j + vx] - mu[j];
              ss[j] = fmaf(d, d, ss[j]);
            }
        }
#pragma unroll
      for (int j = 0; j < PX; ++j) {
        if (x0 + j > nx - kBW) continue;
        const bool inm = ((allm >> j) & 0xFu) == 0xFu;
        out[o + j] = make_float2(mu[j], inm ? ss[j] : -ss[j] - 0.0f);
      }
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
    if (hi > a.nx - kBW) hi = a.nx - kBW;
    unsigned v = 1;
    const uint8_t *row = a.smask + yz * a.nx;
    for (int x = lo; x <= hi + kBW - 1; ++x) v &= row[x] != 0 ? 1u : 0u;
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
    if (hi > a.ny - kBW) hi = a.ny - kBW;
    unsigned v = 1;
    for (int y = lo; y <= hi + kBW - 1; ++y) v &= in[((long long)z * a.ny + y) * a.nbx + bx];
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
    if (hi > a.nz - kBW) hi = a.nz - kBW;
    unsigned v = 1;
    for (int z = lo; z <= hi + kBW - 1; ++z) v &= in[(long long)z * a.nbx * a.nby + bxy];
    out[b] = (uint8_t)v;
  }
}
__device__ __forceinline__ const uint8_t *wand_of(const Args16 &a) {
  return a.wand + (long long)a.nbx * a.ny * a.nz + (long long)a.nbx * a.nby * a.nz;
}

// ---------------------------------------------------------------------------
// Base-block preparation, one thread per block: the FP32 mean, the masked
// sums of x~ and x~^2, the base-mask mode and the two 16-bit parts of x~
// (packed per (part, vz, vy) as two 32-bit words).  grid.y = call.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) prep16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active) return;
  const T *__restrict__ x = static_cast<const T *>(a.base);
  const uint8_t *__restrict__ mb = a.bmask;
  const int nx = a.nx, ny = a.ny;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < a.nblocks;
       b += (long long)gridDim.x * blockDim.x) {
    int bx, by, bz;
    split3(b, a.nbx, a.nby, bx, by, bz);
    const long long o =
        ((long long)(a.stz + bz * a.G) * ny + (a.sty + by * a.G)) * nx + (a.stx + bx * a.G);
    float v[kB];
    uint64_t mbits = 0;
    float sum = 0.f;
#pragma unroll
    for (int i = 0; i < kB; ++i) {
      const long long q = o + ((long long)(i >> 4) * ny + ((i >> 2) & 3)) * nx + (i & 3);
      v[i] = S16<T>::f(x[q]);
      mbits |= (uint64_t)(mb[q] != 0 ? 1u : 0u) << i;
      sum += v[i];
    }
    const float mu = sum * (1.0f / kB);
    float sxx = 0.f, sxt = 0.f, stc = 0.f;
    uint32_t *xb = a.xs + b * 64;
#pragma unroll
    for (int r = 0; r < 16; ++r) {  // r = vz * 4 + vy
      uint32_t hw[2] = {0u, 0u}, lw[2] = {0u, 0u};
#pragma unroll
      for (int vx = 0; vx < 4; ++vx) {
        const int i = r * 4 + vx;
        const float d = v[i] - mu;
        if ((mbits >> i) & 1u) {
          sxx = fmaf(d, d, sxx);
          sxt += d;
        }
        const T h = S16<T>::t(d);
        const T l = S16<T>::t(d - S16<T>::f(h));
        stc += S16<T>::f(h) + S16<T>::f(l);
        hw[vx >> 1] |= S16<T>::bits(h) << (16 * (vx & 1));
        lw[vx >> 1] |= S16<T>::bits(l) << (16 * (vx & 1));
      }
      xb[r * 2] = hw[0];
      xb[r * 2 + 1] = hw[1];
      xb[32 + r * 2] = lw[0];
      xb[32 + r * 2 + 1] = lw[1];
    }
    Prep16 pp;
    pp.mu = mu;
    pp.sxx = sxx;
    pp.sxt = sxt;
    pp.sxt_tc = stc;
    pp.mmode = mbits == ~0ULL ? 1 : (mbits == 0 ? 2 : 0);
    pp.pad[0] = pp.pad[1] = pp.pad[2] = 0;
    a.prep[b] = pp;
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

// Every selected block of a call without the tensor form to the direct
// search; blocks culled by the variance selection get their culled record.
__global__ void route_all16_kernel(const Args16 *calls) {
  const Args16 &a = calls[blockIdx.y];
  if (!a.active || a.tensor) return;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < a.nblocks;
       b += (long long)gridDim.x * blockDim.x) {
    if (a.selected && !a.selected[b]) {
      int bx, by, bz;
      split3(b, a.nbx, a.nby, bx, by, bz);
      const long long orig = ((long long)(a.stz + bz * a.G) * a.ny + (a.sty + by * a.G)) * a.nx +
                             (a.stx + bx * a.G);
      write_out(a, b, -3.f, -3.f, orig, 0);
    } else {
      const unsigned int k = atomicAdd(&a.ctl[1], 1u);
      a.fb_list[k] = (int)b;
    }
  }
}

struct TcMaps {
  CUtensorMap m[kMaxCalls];
};

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

// ---------------------------------------------------------------------------
// The tensor-core search.  Persistent CTAs of 8 warps, three per SM (while
// one waits on memory or on its MMAs the others work).  Row m = 32 (w % 4) +
// lane of A and D is (blk = m / 16, shift s = (m / 2) % 8, part = m % 2);
// warps 0-3 write the A band of k-step 0 and read D columns 0-31 (dz 0-3),
// warps 4-7 k-step 1 and columns 32-63.  A streams through two 32 KB buffers,
// one vz (8 operands) at a time: the CUDA cores write the next vz's bands
// while the tensor cores multiply the previous one.
// ---------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(kThreads, kCtasPerSM)
    ncc_tc_kernel(const Args16 *calls, int ncalls, long long total_tiles,
                  const __grid_constant__ TcMaps maps) {
  static_assert(W >= 2 && W <= 8, "window of the tensor form");
  constexpr int R = W / 2;
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t *const sbase = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(dsm) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t *const sa = sbase;                         // A: 2 buffers of one vz's 8 operands
  uint8_t *const win = sbase + 2 * kAChunkBytes;      // B: the window box
  __shared__ __align__(8) uint64_t s_tma_bar, s_mma_bar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_any, s_fail;
  __shared__ long long s_b[kTileBlocks];
  __shared__ int s_elig[kTileBlocks];
  __shared__ float s_sxx[kTileBlocks], s_stc[kTileBlocks];
  __shared__ Top2 s_part[kTileBlocks];
  __shared__ unsigned int s_cnt[kTileBlocks];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3, half = warp >> 2;
  const int m = 32 * q + lane;            // row of A and D (tensor-memory lane)
  const int blk = m >> 4, sft = (m >> 1) & 7, part = m & 1;

  if (tid == 0) {
    mbar_init(&s_tma_bar, 1);
    mbar_init(&s_mma_bar[0], 1);
    mbar_init(&s_mma_bar[1], 1);
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
  for (int i = tid; i < 2 * kAChunkBytes / 16; i += kThreads)
    reinterpret_cast<uint4 *>(sa)[i] = make_uint4(0u, 0u, 0u, 0u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t lane_addr = tmem + ((uint32_t)(32 * q) << 16);
  // this row's band in k-step `half`: element t0 of the step holds x~[0]
  // (words floor(t0 / 2) ..; an odd t0 straddles the 16-bit halves)
  int t0 = 0;
  // byte offset of 32-bit word c of this row in step r: r * 4 KB + row_off + c_off(c)
  const uint32_t row_off = (uint32_t)(m >> 3) * kASBO + (uint32_t)(m & 7) * 16u;

  unsigned tma_phase = 0, mma_phase[2] = {0u, 0u};
  int cur_call = -1;
  Args16 a;
  for (long long tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    const int ci = call_of_tile(calls, ncalls, tile);
    if (ci != cur_call) {
      a = calls[ci];
      cur_call = ci;
      t0 = a.G * blk + sft - 16 * half;
    }
    const long long lt = tile - a.tile0;
    const int bxg = (int)(lt % a.tiles_x);
    const int bx0 = bxg * a.bpt;
    const long long rest = lt / a.tiles_x;
    const int by = (int)(rest % a.nby), bz = (int)(rest / a.nby);
    const int oy = a.sty + by * a.G, oz = a.stz + bz * a.G;
    if (tid < kTileBlocks) {
      const int bx = bx0 + tid;
      int e = 0;
      long long b = -1;
      if (tid < a.bpt && bx < a.nbx) {
        b = ((long long)bz * a.nby + by) * a.nbx + bx;
        const int ox = a.stx + bx * a.G;
        const long long orig = ((long long)oz * a.ny + oy) * a.nx + ox;
        const bool sel = !a.selected || a.selected[b];
        const Prep16 pp = a.prep[b];
        if (!sel) {
          write_out(a, b, -3.f, -3.f, orig, 0);
        } else if (pp.mmode == 1 && wand_of(a)[b] && pp.sxx > 0.f) {
          e = 1;
          s_sxx[tid] = pp.sxx;
          s_stc[tid] = pp.sxt_tc;
        } else {
          const unsigned int k = atomicAdd(&a.ctl[1], 1u);
          a.fb_list[k] = (int)b;
        }
      }
      s_b[tid] = b;
      s_elig[tid] = e;
      s_cnt[tid] = 0u;
    }
    __syncthreads();
    if (tid == 0) {
      int any = 0;
      for (int j = 0; j < kTileBlocks; ++j) any |= s_elig[j];
      s_any = any;
    }
    __syncthreads();
    if (!s_any) continue;
    if (tid == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                       smem_u32(&s_tma_bar)),
                   "r"((unsigned)kBoxBytes)
                   : "memory");
      tma_load_4d(win, &maps.m[ci], 0, oy - R, oz - R, (a.G * bx0) >> 3, &s_tma_bar);
    }
    // ---- the block's two 16-bit parts for every (vz, vy), in registers ------
    const bool band = t0 < 16 && t0 + 4 > 0;
    const bool live = band && s_elig[blk] != 0;
    uint2 xw[16];
    {
      const uint32_t *xr = a.xs + (live ? s_b[blk] : 0) * 64 + part * 32;
#pragma unroll
      for (int r = 0; r < 16; ++r)
        xw[r] = live ? *reinterpret_cast<const uint2 *>(xr + 2 * r) : make_uint2(0u, 0u);
    }
    const int c0 = t0 >= 0 ? (t0 >> 1) : -((1 - t0) >> 1);  // floor(t0 / 2)
    const bool odd = t0 & 1;
    constexpr uint32_t idesc = (1u << 4) | (S16<T>::kFmt << 7) | (S16<T>::kFmt << 10) |
                               ((uint32_t)(64 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    // ---- per vz: write the A operands of buffer vz % 2, multiply --------------
    for (int vz = 0; vz < 4; ++vz) {
      const int buf = vz & 1;
      if (vz >= 2) {
        // the multiplies of vz - 2 read this buffer: one thread waits for
        // them, the others at the CTA barrier (no issue slots spent polling)
        if (tid == 0 && !mbar_wait(&s_mma_bar[buf], mma_phase[buf], 1 << 24)) {
          atomicExch(&a.ctl[2], 1u);
          s_fail = 1;
        }
        mma_phase[buf] ^= 1u;
        __syncthreads();
        if (s_fail) break;
      }
      if (band) {
        uint8_t *const cb = sa + (size_t)buf * kAChunkBytes + row_off;
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
          uint8_t *const step = cb + (size_t)(2 * vy + half) * kAStepBytes;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int c = c0 + k;
            if (c >= 0 && c < 8 && (k < 2 || odd))
              *reinterpret_cast<uint32_t *>(step + (c >> 2) * kALBO + (c & 3) * 4) = wv[k];
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      tc_fence_before();
      __syncthreads();
      if (tid == 0 && !s_fail) {
        tc_fence_after();
        if (vz == 0 && !mbar_wait(&s_tma_bar, tma_phase, 1 << 22)) {
          s_fail = 1;
          atomicExch(&a.ctl[2], 1u);
        } else {
          const uint32_t wb = smem_u32(win), ab = smem_u32(sa) + (uint32_t)buf * kAChunkBytes;
#pragma unroll 1
          for (int j = 0; j < kAChunkSteps; ++j) {
            const int vy = j >> 1, ks = j & 1;
            const uint64_t ad = sdesc(ab + (uint32_t)j * kAStepBytes, kALBO, kASBO);
            const uint64_t bd = sdesc(wb + (uint32_t)(2 * ks) * kLBO + (uint32_t)vz * kSBO +
                                          (uint32_t)vy * 16u,
                                      kLBO, kSBO);
            const int acc = (vz | j) != 0;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                : "memory");
          }
          asm volatile(
              "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                  smem_u32(&s_mma_bar[buf]))
              : "memory");
        }
      }
      __syncthreads();
      if (s_fail) break;  // every thread sees the same flag
    }
    if (s_fail) break;
    tma_phase ^= 1u;
    // ---- epilogue: the last two commits (vz 2 and 3) ------------------------
    if (tid == 0) {
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
        if (!mbar_wait(&s_mma_bar[bb], mma_phase[bb], 1 << 24)) {
          atomicExch(&a.ctl[2], 1u);
          s_fail = 1;
        }
    }
    mma_phase[0] ^= 1u;
    mma_phase[1] ^= 1u;
    __syncthreads();
    if (s_fail) break;
    tc_fence_after();
    uint32_t d[32];
    tmem_ld32(lane_addr + (uint32_t)(32 * half), d);
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    // add the two parts: part 0 keeps columns 0-15 of this half, part 1 16-31
    float v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const float mine = __uint_as_float(part ? d[16 + j] : d[j]);
      const float send = __uint_as_float(part ? d[j] : d[16 + j]);
      v[j] = mine + __shfl_xor_sync(0xffffffffu, send, 1);
    }
    Top2 tp;
    tp.b1 = -3.f;
    tp.b2 = -3.f;
    tp.i1 = 0x7fffffffffffffffLL;
    unsigned int cnt = 0;
    if (s_elig[blk] && sft < W) {
      const int ox = a.stx + (bx0 + blk) * a.G;
      const int cx = ox - R + sft;
      int xlo, xhi, ylo, yhi, zlo, zhi;
      cand_range(ox, a.nx, W, xlo, xhi);
      cand_range(oy, a.ny, W, ylo, yhi);
      cand_range(oz, a.nz, W, zlo, zhi);
      const float sxx = s_sxx[blk], stc = s_stc[blk];
      if (cx >= xlo && cx <= xhi) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int dz = 4 * half + 2 * part + (j >> 3), py = j & 7;
          const int cy = oy - R + py, cz = oz - R + dz;
          if (py < W && dz < W && cy >= ylo && cy <= yhi && cz >= zlo && cz <= zhi) {
            const long long idx = ((long long)cz * a.ny + cy) * a.nx + cx;
            const float2 st = __ldg(a.stats + idx);
            const float sxy = v[j] - st.x * stc;
            const float syy = st.y;
            const float sc = syy > 0.f ? __fdividef(sxy * sxy, sxx * syy) : -2.f;
            top2_add(tp, sc, idx);
            ++cnt;
          }
        }
      }
    }
    // reduce over the 16 lanes of the block (8 shifts x 2 parts) ...
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) top2_merge(tp, top2_shfl_xor(tp, o));
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    // ... then over the two halves of the candidate planes
    if (half == 1 && (lane & 15) == 0) {
      s_part[blk] = tp;
      s_cnt[blk] = cnt;
    }
    tc_fence_before();
    __syncthreads();
    if (half == 0 && (lane & 15) == 0 && s_elig[blk]) {
      top2_merge(tp, s_part[blk]);
      cnt += s_cnt[blk];
      write_out(a, s_b[blk], tp.b1, tp.b2, tp.i1, 1);
      atomicAdd(&a.ctl[0], 1u);
      if (a.ncc_count) atomicAdd(a.ncc_count, (unsigned long long)cnt);
    }
    if (s_fail) break;
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
// call's fb_list): one CTA per block, candidates over the threads, the masked
// sums of the reference formula per candidate.  A candidate whose footprint
// lies inside the search mask with the base block inside its mask uses the
// box statistics for Syy and one product per voxel.  grid.y = call.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) ncc_fb16_kernel(const Args16 *calls) {
  constexpr int NT = 128;
  __shared__ float s_xt[kB], s_mb[kB];
  __shared__ float s_y[16 * 16 * 16];
  __shared__ uint8_t s_m[16 * 16 * 16];
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
    cand_range(ox, a.nx, a.W, xlo, xhi);
    cand_range(oy, a.ny, a.W, ylo, yhi);
    cand_range(oz, a.nz, a.W, zlo, zhi);
    const int ncx = xhi - xlo + 1, ncy = yhi - ylo + 1, ncz = zhi - zlo + 1;
    const int ex = ncx + kBW - 1, ey = ncy + kBW - 1, ez = ncz + kBW - 1;
    const Prep16 pp = a.prep[b];
    __syncthreads();
    if (tid < kB) {
      const int vx = tid & 3, vy = (tid >> 2) & 3, vz = tid >> 4;
      const long long qq = ((long long)(oz + vz) * a.ny + (oy + vy)) * a.nx + (ox + vx);
      const float mv = a.bmask[qq] != 0 ? 1.f : 0.f;
      s_xt[tid] = S16<T>::f(base[qq]) - pp.mu;
      s_mb[tid] = mv;
    }
    for (int i = tid; i < ex * ey * ez; i += NT) {
      const int wx = i % ex, wy = (i / ex) % ey, wz = i / (ex * ey);
      const long long qq = ((long long)(zlo + wz) * a.ny + (ylo + wy)) * a.nx + (xlo + wx);
      s_y[(wz * 16 + wy) * 16 + wx] = S16<T>::f(search[qq]);
      s_m[(wz * 16 + wy) * 16 + wx] = a.smask[qq] != 0 ? 1 : 0;
    }
    __syncthreads();
    Top2 tp;
    tp.b1 = -3.f;
    tp.b2 = -3.f;
    tp.i1 = 0x7fffffffffffffffLL;
    const int nc = ncx * ncy * ncz;
    for (int c = tid; c < nc; c += NT) {
      const int px = c % ncx, py = (c / ncx) % ncy, pz = c / (ncx * ncy);
      const int cx = xlo + px, cy = ylo + py, cz = zlo + pz;
      const long long idx = ((long long)cz * a.ny + cy) * a.nx + cx;
      const float2 st = __ldg(a.stats + idx);
      const float muy = st.x;
      float sxy = 0.f, sxx = 0.f, syy = 0.f;
      if (pp.mmode == 1 && !signbit(st.y)) {
        // footprint and base block wholly inside their masks
#pragma unroll 8
        for (int i = 0; i < kB; ++i) {
          const int vx = i & 3, vy = (i >> 2) & 3, vz = i >> 4;
          sxy = fmaf(s_xt[i], s_y[((pz + vz) * 16 + py + vy) * 16 + px + vx], sxy);
        }
        sxy -= muy * pp.sxt;
        sxx = pp.sxx;
        syy = st.y;
      } else {
#pragma unroll 8
        for (int i = 0; i < kB; ++i) {
          const int vx = i & 3, vy = (i >> 2) & 3, vz = i >> 4;
          const int w = ((pz + vz) * 16 + py + vy) * 16 + px + vx;
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

size_t tc_smem_bytes() { return (size_t)2 * kAChunkBytes + kBoxBytes + 1024; }

}  // namespace

// Derived per-call fields: the tensor form's tile layout and copy geometry.
void prepare16(const BmGeom &g, Match16Call &c) {
  c.nx = g.size[0]; c.ny = g.size[1]; c.nz = g.size[2];
  c.nbx = g.nb[0]; c.nby = g.nb[1]; c.nbz = g.nb[2];
  c.stx = g.st[0]; c.sty = g.st[1]; c.stz = g.st[2];
  c.G = g.ngap;
  c.W = g.nw;
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

size_t match16_wand_bytes(const Match16Call &c) {
  return (size_t)c.nbx * c.ny * c.nz + (size_t)c.nbx * c.nby * c.nz + (size_t)c.nblocks;
}

namespace {

template <typename T>
mirorr_status run16(int ncalls, Match16Call *host_calls, DevBuf &calls_dev, cudaStream_t s) {
  const int SM = sm_count();
  const long long tiles = match16_number_tiles(host_calls, ncalls);
  long long max_vox = 0, max_blocks = 0, max_chunks = 0;
  int W = 0, G = 0;
  bool any_tensor = false;
  for (int i = 0; i < ncalls; ++i) {
    const Match16Call &c = host_calls[i];
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
  box_stats16_kernel<T><<<grid_for(max_vox / 4 + 1), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  wand_x16_kernel<<<grid_for(max_vox / 2 + 1), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  wand_y16_kernel<<<grid_for(max_vox / 4 + 1), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  wand_z16_kernel<<<grid_for(max_blocks), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  prep16_kernel<T><<<grid_for(max_blocks), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  if (any_tensor) {
    chunk16_kernel<T><<<grid_for(max_chunks), 256, 0, s>>>(dc);
    MB2_LAUNCH_CHECK();
  }
  route_all16_kernel<<<grid_for(max_blocks), 256, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  if (any_tensor) {
    if (ncalls > kMaxCalls) {
      set_error("more than %d matcher calls in one tensor launch", kMaxCalls);
      return MIRORR_EINVAL;
    }
    EncodeTiledFn enc = encode_fn();
    if (!enc) {
      set_error("cuTensorMapEncodeTiled is not available from the driver");
      return MIRORR_ECUDA;
    }
    static TcMaps maps;  // the host side of the kernel parameter (large: static)
    static std::mutex maps_mu;
    std::lock_guard<std::mutex> lock(maps_mu);
    memset(&maps, 0, sizeof(maps));
    for (int i = 0; i < ncalls; ++i) {
      const Match16Call &c = host_calls[i];
      if (!c.active || !c.tensor) continue;
      const cuuint64_t dims[4] = {8, (cuuint64_t)c.ny, (cuuint64_t)c.nz, (cuuint64_t)c.nxc};
      const cuuint64_t strides[3] = {16, (cuuint64_t)16 * c.ny, (cuuint64_t)16 * c.ny * c.nz};
      const cuuint32_t box[4] = {8, (cuuint32_t)kSlots, (cuuint32_t)kPlanes, (cuuint32_t)kXC};
      const cuuint32_t estr[4] = {1, 1, 1, 1};
      CUresult r = enc(&maps.m[i],
                       S16<T>::kFmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                       4, c.chunked, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return MIRORR_ECUDA;
      }
    }
    const size_t smem = tc_smem_bytes();
    auto kern = (W == 7) ? ncc_tc_kernel<T, 7> : (W == 5) ? ncc_tc_kernel<T, 5>
                                                          : ncc_tc_kernel<T, 3>;
    MB2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long grid = tiles < (long long)SM * kCtasPerSM ? tiles : (long long)SM * kCtasPerSM;
    if (grid > 0) {
      kern<<<(unsigned)grid, kThreads, smem, s>>>(dc, ncalls, tiles, maps);
      MB2_LAUNCH_CHECK();
    }
  }
  ncc_fb16_kernel<T><<<dim3((unsigned)SM * 4, (unsigned)ncalls), 128, 0, s>>>(dc);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace

mirorr_status launch_match16_batch(int dtype, int ncalls, Match16Call *host_calls,
                                   DevBuf &calls_dev, cudaStream_t s) {
  if (ncalls <= 0) return MIRORR_OK;
  if (dtype == MIRORR_DTYPE_BF16) return run16<__nv_bfloat16>(ncalls, host_calls, calls_dev, s);
  if (dtype == MIRORR_DTYPE_F16) return run16<__half>(ncalls, host_calls, calls_dev, s);
  set_error("storage type %d is not a 16-bit type", dtype);
  return MIRORR_EINVAL;
}

mirorr_status launch_match16(int dtype, const BmGeom &g, const void *base, const uint8_t *bmask,
                             const void *search, const uint8_t *smask, const uint8_t *selected,
                             const BmOut &out, Bm16Work &w, unsigned long long *ncc_count,
                             cudaStream_t s) {
  if (g.bw != kBW) {
    set_error("the 16-bit search supports block width 4 (got %d)", g.bw);
    return MIRORR_EINVAL;
  }
  if (g.bgap != 1) {
    set_error("the 16-bit search supports block gap 1 (got %d)", g.bgap);
    return MIRORR_EINVAL;
  }
  if (g.nw > 13) {
    set_error("the 16-bit search supports windows up to 13 (got %d)", g.nw);
    return MIRORR_EINVAL;
  }
  Match16Call c;
  memset(&c, 0, sizeof(c));
  prepare16(g, c);
  const long long nvox = (long long)g.size[0] * g.size[1] * g.size[2];
  MB2_TRY(w.stats.ensure(sizeof(float2) * nvox));
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
