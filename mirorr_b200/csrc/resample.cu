// resample.cu -- linear resampler and pyramid smoothing for sm_100a.
//
// Resampler: itk::ResampleImageFilter driven by itk::LinearInterpolateImageFunction
// (call sites itkMirorrRegistrationMethod.txx:523-570,603-604,
// itkSymMirorrRegistrationMethod.txx:388-437,481-484), restated:
//   * the output index maps to the input continuous index c = e + C idx,
//     evaluated left to right in FP64 without contraction;
//   * inside test -0.5 <= c < n - 0.5 (ITK's centred-pixel buffer test),
//     otherwise the default value 0;
//   * neighbour indices clamp to the image (a neighbour past the last voxel
//     repeats the base voxel) and non-positive distances contribute nothing;
//   * lerp chain x -> y -> z, a + (b - a) t, in FP64;
//   * float output rounded to nearest; uint8 output clamped to [0, 255] and
//     truncated (ResampleImageFilter::CastPixelWithBoundsChecking).
// An image and its mask on the same input grid go through one launch, which
// computes each voxel's index map once for both.
// The FP64 arithmetic is written with explicit round-to-nearest intrinsics so
// results are bit-identical to a plain C evaluation of the same expressions.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "kernels.cuh"

namespace mb2 {

struct ResampleArgs {
  const void *in;  // float32, or 16-bit (kernel template type)
  const uint8_t *inm;
  int inx, iny, inz;
  int onx, ony, onz;
  double C[9];
  double e[3];
  void *out;       // float32, or 16-bit
  uint8_t *outm;
  int nearest;    // nearest-neighbour instead of linear interpolation
  int mask_ones;  // the input mask is 255 everywhere: the output mask is 255
                  // inside the input and 0 outside (every interpolation of
                  // 255s is 255), so the mask is not read
};

__device__ __forceinline__ float ld_f(const float *p, long long i) { return __ldg(p + i); }
__device__ __forceinline__ float ld_f(const __nv_bfloat16 *p, long long i) {
  return __bfloat162float(p[i]);
}
__device__ __forceinline__ float ld_f(const __half *p, long long i) { return __half2float(p[i]); }
// An interpolated FP64 value as stored: rounded to float, then (16-bit
// storage) rounded again to the storage type.
__device__ __forceinline__ void st_v(float &d, double v) { d = __double2float_rn(v); }
__device__ __forceinline__ void st_v(__nv_bfloat16 &d, double v) {
  d = __float2bfloat16_rn(__double2float_rn(v));
}
__device__ __forceinline__ void st_v(__half &d, double v) {
  d = __float2half_rn(__double2float_rn(v));
}
__device__ __forceinline__ void st_copy(float &d, float v) { d = v; }
__device__ __forceinline__ void st_copy(__nv_bfloat16 &d, float v) { d = __float2bfloat16_rn(v); }
__device__ __forceinline__ void st_copy(__half &d, float v) { d = __float2half_rn(v); }

__device__ inline double dlerp(double a, double b, double t) {
  return __dadd_rn(a, __dmul_rn(__dsub_rn(b, a), t));
}

// Linear or nearest resampling of one output voxel (i, j, k); cj, ck hold
// C[r][1] * j and C[r][2] * k (products the whole x-run shares).  Writes the
// image value to *v and the mask value to *m when the respective input exists.
template <bool IMG, bool MSK, typename TI, typename TO>
__device__ __forceinline__ void resample_voxel(const ResampleArgs &a, int i, const double cj[3],
                                               const double ck[3], TO *v, uint8_t *m) {
  const TI *in = static_cast<const TI *>(a.in);
  const double di = (double)i;
  double c[3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
    c[r] = __dadd_rn(__dadd_rn(__dadd_rn(a.e[r], __dmul_rn(a.C[3 * r], di)), cj[r]), ck[r]);
  const int nn[3] = {a.inx, a.iny, a.inz};
  bool inside = true;
#pragma unroll
  for (int r = 0; r < 3; ++r)
    if (!(c[r] >= -0.5 && c[r] < (double)nn[r] - 0.5)) inside = false;
  const bool mread = MSK && !a.mask_ones;
  if (a.nearest) {
    if (!inside) {
      if (IMG) st_copy(*v, 0.0f);
      if (MSK) *m = 0;
      return;
    }
    if (MSK && a.mask_ones) *m = 255;
    // NearestNeighborInterpolateImageFunction: index = floor(c + 0.5)
    long long q = 0, stride = 1;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      int b = (int)floor(__dadd_rn(c[r], 0.5));
      if (b < 0) b = 0;
      if (b > nn[r] - 1) b = nn[r] - 1;
      q += (long long)b * stride;
      stride *= nn[r];
    }
    if (IMG) st_copy(*v, ld_f(in, q));
    if (mread) *m = __ldg(a.inm + q);
    return;
  }
  if (!IMG && !mread) {
    if (MSK) *m = inside ? 255 : 0;
    return;
  }
  // Linear: every voxel is evaluated, with its neighbours clamped into the
  // image (straight-line code, so the voxels of a run overlap), and the
  // inside test selects the result.  Inside the image the clamps change
  // nothing: floor(c) lies in [-1, n - 1].
  int i0[3], i1[3];
  double t[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double cc = fmin(fmax(c[r], -1.0), (double)nn[r]);  // NaN -> -1
    int b = (int)floor(cc);
    b = b < 0 ? 0 : (b > nn[r] - 1 ? nn[r] - 1 : b);
    double d = __dsub_rn(c[r], (double)b);
    if (d <= 0.0) d = 0.0;
    i0[r] = b;
    i1[r] = (b + 1 > nn[r] - 1) ? b : b + 1;
    t[r] = d;
  }
  // the eight neighbours: a base pointer and 32-bit deltas (a slice holds
  // fewer than 2^31 voxels, checked by the launcher)
  const int sy = a.inx, sz = a.inx * a.iny;
  const long long q000 = (long long)i0[2] * sz + (long long)(i0[1] * sy + i0[0]);
  const int dx = i1[0] - i0[0], dy = (i1[1] - i0[1]) * sy, dz = (i1[2] - i0[2]) * sz;
  if (IMG) {
    const TI *p = in + q000;
    const double x00 = dlerp((double)ld_f(p, 0), (double)ld_f(p, dx), t[0]);
    const double x10 = dlerp((double)ld_f(p, dy), (double)ld_f(p, dy + dx), t[0]);
    const double x01 = dlerp((double)ld_f(p, dz), (double)ld_f(p, dz + dx), t[0]);
    const double x11 = dlerp((double)ld_f(p, dz + dy), (double)ld_f(p, dz + dy + dx), t[0]);
    const double val = dlerp(dlerp(x00, x10, t[1]), dlerp(x01, x11, t[1]), t[2]);
    st_v(*v, inside ? val : 0.0);
  }
  if (MSK && !mread) *m = inside ? 255 : 0;
  if (mread) {
    const uint8_t *p = a.inm + q000;
    const uint8_t m000 = __ldg(p), m100 = __ldg(p + dx), m010 = __ldg(p + dy),
                  m110 = __ldg(p + dy + dx), m001 = __ldg(p + dz), m101 = __ldg(p + dz + dx),
                  m011 = __ldg(p + dz + dy), m111 = __ldg(p + dz + dy + dx);
    if (!inside) {
      *m = 0;
    } else if (m000 == m100 && m000 == m010 && m000 == m110 && m000 == m001 && m000 == m101 &&
               m000 == m011 && m000 == m111) {
      // every lerp of equal values returns that value exactly
      *m = m000;
    } else {
      const double x00 = dlerp((double)m000, (double)m100, t[0]);
      const double x10 = dlerp((double)m010, (double)m110, t[0]);
      const double x01 = dlerp((double)m001, (double)m101, t[0]);
      const double x11 = dlerp((double)m011, (double)m111, t[0]);
      double w = dlerp(dlerp(x00, x10, t[1]), dlerp(x01, x11, t[1]), t[2]);
      if (w < 0.0) w = 0.0;
      if (w > 255.0) w = 255.0;
      *m = (uint8_t)(int)w;
    }
  }
}

// Each thread produces a run of 4 consecutive output voxels (linear order, so
// a run may cross a row) and stores them with one 16-byte image store and one
// 4-byte mask store.  The output buffers are 16-byte aligned (checked by the
// launcher).  Per voxel the index map is the same FP64 expression as a plain
// evaluation; only the j and k products are shared along the run.
template <bool IMG, bool MSK, typename TI, typename TO>
__device__ __forceinline__ void resample_runs(const ResampleArgs &a, long long g0, long long gstride) {
  TO *const out = static_cast<TO *>(a.out);
  const long long n = (long long)a.onx * a.ony * a.onz;
  const long long nrun = (n + 3) >> 2;
  const bool narrow = n < (1LL << 31);
  const bool row_runs = (a.onx & 3) == 0;  // then no run crosses a row
  for (long long g = g0; g < nrun; g += gstride) {
    const long long o0 = g << 2;
    int i, j, k;
    if (narrow) {
      // 32-bit division (the output holds fewer than 2^31 voxels)
      const unsigned int u = (unsigned int)o0, onx = (unsigned int)a.onx;
      const unsigned int row = u / onx;
      i = (int)(u - row * onx);
      j = (int)(row % (unsigned int)a.ony);
      k = (int)(row / (unsigned int)a.ony);
    } else {
      split3(o0, a.onx, a.ony, i, j, k);
    }
    double cj[3], ck[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      cj[r] = __dmul_rn(a.C[3 * r + 1], (double)j);
      ck[r] = __dmul_rn(a.C[3 * r + 2], (double)k);
    }
    TO v[4];
    uint8_t m[4] = {0, 0, 0, 0};
    const int cnt = n - o0 < 4 ? (int)(n - o0) : 4;
    if (row_runs) {
      // the run lies in one row: four independent voxels
#pragma unroll
      for (int u = 0; u < 4; ++u) resample_voxel<IMG, MSK, TI, TO>(a, i + u, cj, ck, &v[u], &m[u]);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        st_copy(v[u], 0.0f);
        if (u < cnt) {
          resample_voxel<IMG, MSK, TI, TO>(a, i, cj, ck, &v[u], &m[u]);
          if (++i == a.onx) {
            i = 0;
            if (++j == a.ony) {
              j = 0;
              ++k;
#pragma unroll
              for (int r = 0; r < 3; ++r) ck[r] = __dmul_rn(a.C[3 * r + 2], (double)k);
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) cj[r] = __dmul_rn(a.C[3 * r + 1], (double)j);
          }
        }
      }
    }
    if (cnt == 4) {
      if (IMG) {
        if (sizeof(TO) == 4) {
          *reinterpret_cast<float4 *>(out + o0) =
              make_float4(*reinterpret_cast<float *>(&v[0]), *reinterpret_cast<float *>(&v[1]),
                          *reinterpret_cast<float *>(&v[2]), *reinterpret_cast<float *>(&v[3]));
        } else {
          const unsigned short *h = reinterpret_cast<const unsigned short *>(v);
          *reinterpret_cast<uint2 *>(out + o0) =
              make_uint2((uint32_t)h[0] | ((uint32_t)h[1] << 16), (uint32_t)h[2] | ((uint32_t)h[3] << 16));
        }
      }
      if (MSK)
        *reinterpret_cast<uint32_t *>(a.outm + o0) =
            (uint32_t)m[0] | ((uint32_t)m[1] << 8) | ((uint32_t)m[2] << 16) | ((uint32_t)m[3] << 24);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (u < cnt) {
          if (IMG) out[o0 + u] = v[u];
          if (MSK) a.outm[o0 + u] = m[u];
        }
      }
    }
  }
}

// resident CTAs of 256 threads per SM the resampling kernels are compiled for
#ifndef MB2_RS_MINB
#define MB2_RS_MINB 3
#endif

template <bool IMG, bool MSK, typename TI, typename TO>
__global__ void __launch_bounds__(256, MB2_RS_MINB) resample_kernel(ResampleArgs a) {
  resample_runs<IMG, MSK, TI, TO>(a, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                                  (long long)gridDim.x * blockDim.x);
}

// Many resampling passes in one launch (grid.y = job).  A job's image is
// float32 in and `out_dtype` out (or absent: mask only).
__global__ void __launch_bounds__(256, MB2_RS_MINB) resample_batch_kernel(const ResampleJob *jobs) {
  const ResampleJob &j = jobs[blockIdx.y];
  if (!j.active) return;
  ResampleArgs a;
  a.in = j.in; a.inm = j.inm;
  a.inx = j.in_size[0]; a.iny = j.in_size[1]; a.inz = j.in_size[2];
  a.onx = j.out_size[0]; a.ony = j.out_size[1]; a.onz = j.out_size[2];
#pragma unroll
  for (int i = 0; i < 9; ++i) a.C[i] = j.C[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) a.e[i] = j.e[i];
  a.out = j.out; a.outm = j.outm; a.nearest = 0; a.mask_ones = j.mask_ones;
  const long long g0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long gs = (long long)gridDim.x * blockDim.x;
  if (!a.in || !a.out) {
    resample_runs<false, true, float, float>(a, g0, gs);
  } else if (a.inm && a.outm) {
    if (j.out_dtype == MIRORR_DTYPE_BF16) resample_runs<true, true, float, __nv_bfloat16>(a, g0, gs);
    else if (j.out_dtype == MIRORR_DTYPE_F16) resample_runs<true, true, float, __half>(a, g0, gs);
    else resample_runs<true, true, float, float>(a, g0, gs);
  } else {
    a.inm = nullptr;
    a.outm = nullptr;
    if (j.out_dtype == MIRORR_DTYPE_BF16) resample_runs<true, false, float, __nv_bfloat16>(a, g0, gs);
    else if (j.out_dtype == MIRORR_DTYPE_F16) resample_runs<true, false, float, __half>(a, g0, gs);
    else resample_runs<true, false, float, float>(a, g0, gs);
  }
}

mirorr_status launch_resample_batch(const ResampleJob *dev_jobs, int njobs, long long max_voxels,
                                    cudaStream_t s) {
  if (njobs <= 0) return MIRORR_OK;
  long long blocks = ((max_voxels + 3) / 4 + 255) / 256;
  const long long cap = (long long)sm_count() * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  resample_batch_kernel<<<dim3((unsigned)blocks, njobs), 256, 0, s>>>(dev_jobs);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

template <typename TI, typename TO>
void launch_rs(const ResampleArgs &a, unsigned blocks, cudaStream_t s) {
  if (a.out && a.outm) resample_kernel<true, true, TI, TO><<<blocks, 256, 0, s>>>(a);
  else if (a.out) resample_kernel<true, false, TI, TO><<<blocks, 256, 0, s>>>(a);
  else resample_kernel<false, true, float, float><<<blocks, 256, 0, s>>>(a);
}

mirorr_status launch_resample(const int in_size[3], const void *in, const uint8_t *in_mask,
                              const int out_size[3], const ResampleMap &map, void *out,
                              uint8_t *out_mask, cudaStream_t s, bool nearest, int in_dtype,
                              int out_dtype, bool mask_ones) {
  ResampleArgs a;
  a.nearest = nearest ? 1 : 0;
  a.mask_ones = mask_ones ? 1 : 0;
  a.in = in; a.inm = in_mask;
  a.inx = in_size[0]; a.iny = in_size[1]; a.inz = in_size[2];
  a.onx = out_size[0]; a.ony = out_size[1]; a.onz = out_size[2];
  for (int i = 0; i < 9; ++i) a.C[i] = map.C[i];
  for (int i = 0; i < 3; ++i) a.e[i] = map.e[i];
  a.out = in ? out : nullptr;
  a.outm = in_mask ? out_mask : nullptr;
  long long n = (long long)out_size[0] * out_size[1] * out_size[2];
  if (n <= 0 || (!a.out && !a.outm)) return MIRORR_OK;
  if (((uintptr_t)a.out & 15u) || ((uintptr_t)a.outm & 3u)) {
    set_error("resampler output buffers must be 16-byte (image) and 4-byte (mask) aligned");
    return MIRORR_EINVAL;
  }
  if ((long long)in_size[0] * in_size[1] >= (1LL << 31)) {
    set_error("resampler input slice of %d x %d voxels: at most 2^31 - 1", in_size[0], in_size[1]);
    return MIRORR_EINVAL;
  }
  long long blocks = ((n + 3) / 4 + 255) / 256;
  const long long cap = (long long)sm_count() * 8;
  if (blocks > cap) blocks = cap;
  const unsigned nb = (unsigned)blocks;
  if (!a.out || (in_dtype == MIRORR_DTYPE_F32 && out_dtype == MIRORR_DTYPE_F32)) {
    launch_rs<float, float>(a, nb, s);
  } else if (out_dtype == MIRORR_DTYPE_BF16 && in_dtype == MIRORR_DTYPE_F32) {
    launch_rs<float, __nv_bfloat16>(a, nb, s);
  } else if (out_dtype == MIRORR_DTYPE_BF16 && in_dtype == MIRORR_DTYPE_BF16) {
    launch_rs<__nv_bfloat16, __nv_bfloat16>(a, nb, s);
  } else if (out_dtype == MIRORR_DTYPE_F16 && in_dtype == MIRORR_DTYPE_F32) {
    launch_rs<float, __half>(a, nb, s);
  } else if (out_dtype == MIRORR_DTYPE_F16 && in_dtype == MIRORR_DTYPE_F16) {
    launch_rs<__half, __half>(a, nb, s);
  } else {
    set_error("resampler type pair %d -> %d not supported", in_dtype, out_dtype);
    return MIRORR_EINVAL;
  }
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

// Separable Gaussian pass: FP64 accumulation in tap order, clamp-to-edge,
// float output (the input of the first pass may be 16-bit).
template <typename TI>
__global__ void smooth_axis_kernel(const TI *__restrict__ in, float *__restrict__ out, int nx,
                                   int ny, int nz, int axis, const double *__restrict__ w,
                                   int radius) {
  long long n = (long long)nx * ny * nz;
  const int len = axis == 0 ? nx : (axis == 1 ? ny : nz);
  const long long stride = axis == 0 ? 1 : (axis == 1 ? nx : (long long)nx * ny);
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    int pos = axis == 0 ? (int)(o % nx) : (axis == 1 ? (int)((o / nx) % ny) : (int)(o / ((long long)nx * ny)));
    long long base = o - (long long)pos * stride;
    double acc = 0.0;
    for (int t = 0; t <= 2 * radius; ++t) {
      int q = pos + t - radius;
      q = q < 0 ? 0 : (q > len - 1 ? len - 1 : q);
      acc = __dadd_rn(acc, __dmul_rn(w[t], (double)ld_f(in, base + q * stride)));
    }
    out[o] = __double2float_rn(acc);
  }
}

mirorr_status launch_smooth_axis(const int size[3], const void *in, float *out, int axis,
                                 const double *w, int radius, cudaStream_t s, int in_dtype) {
  long long n = (long long)size[0] * size[1] * size[2];
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sm_count() * 64) blocks = (long long)sm_count() * 64;
  if (in_dtype == MIRORR_DTYPE_BF16)
    smooth_axis_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16 *>(in), out,
                                                        size[0], size[1], size[2], axis, w, radius);
  else if (in_dtype == MIRORR_DTYPE_F16)
    smooth_axis_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const __half *>(in), out,
                                                        size[0], size[1], size[2], axis, w, radius);
  else
    smooth_axis_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const float *>(in), out,
                                                        size[0], size[1], size[2], axis, w, radius);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

// float32 -> 16-bit storage (round to nearest even).
template <typename TO>
__global__ void to16_kernel(const float *__restrict__ in, TO *__restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    st_copy(out[i], in[i]);
}

// 16-bit storage -> float32 (exact).
template <typename TI>
__global__ void from16_kernel(const TI *__restrict__ in, float *__restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = ld_f(in, i);
}

mirorr_status launch_from16(const void *in, float *out, long long n, int dtype, cudaStream_t s) {
  if (n <= 0) return MIRORR_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sm_count() * 16) blocks = (long long)sm_count() * 16;
  if (dtype == MIRORR_DTYPE_BF16)
    from16_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16 *>(in), out, n);
  else if (dtype == MIRORR_DTYPE_F16)
    from16_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const __half *>(in), out, n);
  else {
    set_error("storage type %d is not a 16-bit type", dtype);
    return MIRORR_EINVAL;
  }
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

mirorr_status launch_to16(const float *in, void *out, long long n, int dtype, cudaStream_t s) {
  if (n <= 0) return MIRORR_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sm_count() * 16) blocks = (long long)sm_count() * 16;
  if (dtype == MIRORR_DTYPE_BF16)
    to16_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, static_cast<__nv_bfloat16 *>(out), n);
  else if (dtype == MIRORR_DTYPE_F16)
    to16_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, static_cast<__half *>(out), n);
  else {
    set_error("storage type %d is not a 16-bit type", dtype);
    return MIRORR_EINVAL;
  }
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

__global__ void fill_u8_kernel(uint8_t *p, long long n, uint8_t v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

mirorr_status launch_fill_u8(uint8_t *p, long long n, uint8_t v, cudaStream_t s) {
  if (n <= 0) return MIRORR_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sm_count() * 16) blocks = (long long)sm_count() * 16;
  fill_u8_kernel<<<(unsigned)blocks, 256, 0, s>>>(p, n, v);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace mb2
