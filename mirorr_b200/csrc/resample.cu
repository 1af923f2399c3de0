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
// The FP64 arithmetic is written with explicit round-to-nearest intrinsics so
// results are bit-identical to a plain C evaluation of the same expressions.
#include "kernels.cuh"

namespace mb2 {

struct ResampleArgs {
  const float *in;
  const uint8_t *inm;
  int inx, iny, inz;
  int onx, ony, onz;
  double C[9];
  double e[3];
  float *out;
  uint8_t *outm;
  int nearest;  // nearest-neighbour instead of linear interpolation
};

__device__ inline double dlerp(double a, double b, double t) {
  return __dadd_rn(a, __dmul_rn(__dsub_rn(b, a), t));
}

__global__ void __launch_bounds__(256) resample_kernel(ResampleArgs a) {
  long long n = (long long)a.onx * a.ony * a.onz;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    split3(o, a.onx, a.ony, i, j, k);
    const double di = (double)i, dj = (double)j, dk = (double)k;
    double c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
      c[r] = __dadd_rn(__dadd_rn(__dadd_rn(a.e[r], __dmul_rn(a.C[3 * r], di)),
                                 __dmul_rn(a.C[3 * r + 1], dj)),
                       __dmul_rn(a.C[3 * r + 2], dk));
    const int nn[3] = {a.inx, a.iny, a.inz};
    bool inside = true;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (!(c[r] >= -0.5 && c[r] < (double)nn[r] - 0.5)) inside = false;
    if (!inside) {
      if (a.out) a.out[o] = 0.0f;
      if (a.outm) a.outm[o] = 0;
      continue;
    }
    if (a.nearest) {
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
      if (a.out) a.out[o] = __ldg(a.in + q);
      if (a.outm) a.outm[o] = __ldg(a.inm + q);
      continue;
    }
    int i0[3], i1[3];
    double t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      int b = (int)floor(c[r]);
      if (b < 0) b = 0;
      double d = __dsub_rn(c[r], (double)b);
      if (d <= 0.0) d = 0.0;
      i0[r] = b;
      i1[r] = (b + 1 > nn[r] - 1) ? b : b + 1;
      t[r] = d;
    }
    const long long sx = 1, sy = a.inx, sz = (long long)a.inx * a.iny;
    const long long q000 = i0[2] * sz + i0[1] * sy + i0[0] * sx;
    const long long q100 = i0[2] * sz + i0[1] * sy + i1[0] * sx;
    const long long q010 = i0[2] * sz + i1[1] * sy + i0[0] * sx;
    const long long q110 = i0[2] * sz + i1[1] * sy + i1[0] * sx;
    const long long q001 = i1[2] * sz + i0[1] * sy + i0[0] * sx;
    const long long q101 = i1[2] * sz + i0[1] * sy + i1[0] * sx;
    const long long q011 = i1[2] * sz + i1[1] * sy + i0[0] * sx;
    const long long q111 = i1[2] * sz + i1[1] * sy + i1[0] * sx;
    if (a.out) {
      const float *p = a.in;
      double x00 = dlerp((double)__ldg(p + q000), (double)__ldg(p + q100), t[0]);
      double x10 = dlerp((double)__ldg(p + q010), (double)__ldg(p + q110), t[0]);
      double x01 = dlerp((double)__ldg(p + q001), (double)__ldg(p + q101), t[0]);
      double x11 = dlerp((double)__ldg(p + q011), (double)__ldg(p + q111), t[0]);
      double xx0 = dlerp(x00, x10, t[1]);
      double xx1 = dlerp(x01, x11, t[1]);
      a.out[o] = __double2float_rn(dlerp(xx0, xx1, t[2]));
    }
    if (a.outm) {
      const uint8_t *p = a.inm;
      double x00 = dlerp((double)__ldg(p + q000), (double)__ldg(p + q100), t[0]);
      double x10 = dlerp((double)__ldg(p + q010), (double)__ldg(p + q110), t[0]);
      double x01 = dlerp((double)__ldg(p + q001), (double)__ldg(p + q101), t[0]);
      double x11 = dlerp((double)__ldg(p + q011), (double)__ldg(p + q111), t[0]);
      double xx0 = dlerp(x00, x10, t[1]);
      double xx1 = dlerp(x01, x11, t[1]);
      double v = dlerp(xx0, xx1, t[2]);
      if (v < 0.0) v = 0.0;
      if (v > 255.0) v = 255.0;
      a.outm[o] = (uint8_t)(int)v;
    }
  }
}

mirorr_status launch_resample(const int in_size[3], const float *in, const uint8_t *in_mask,
                              const int out_size[3], const ResampleMap &map, float *out,
                              uint8_t *out_mask, cudaStream_t s, bool nearest) {
  ResampleArgs a;
  a.nearest = nearest ? 1 : 0;
  a.in = in; a.inm = in_mask;
  a.inx = in_size[0]; a.iny = in_size[1]; a.inz = in_size[2];
  a.onx = out_size[0]; a.ony = out_size[1]; a.onz = out_size[2];
  for (int i = 0; i < 9; ++i) a.C[i] = map.C[i];
  for (int i = 0; i < 3; ++i) a.e[i] = map.e[i];
  a.out = in ? out : nullptr;
  a.outm = in_mask ? out_mask : nullptr;
  long long n = (long long)out_size[0] * out_size[1] * out_size[2];
  if (n <= 0) return MIRORR_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  resample_kernel<<<(unsigned)blocks, 256, 0, s>>>(a);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

// Separable Gaussian pass: FP64 accumulation in tap order, clamp-to-edge,
// float output.
__global__ void smooth_axis_kernel(const float *__restrict__ in, float *__restrict__ out, int nx,
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
      acc = __dadd_rn(acc, __dmul_rn(w[t], (double)__ldg(&in[base + q * stride])));
    }
    out[o] = __double2float_rn(acc);
  }
}

mirorr_status launch_smooth_axis(const int size[3], const float *in, float *out, int axis,
                                 const double *w, int radius, cudaStream_t s) {
  long long n = (long long)size[0] * size[1] * size[2];
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  smooth_axis_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, out, size[0], size[1], size[2], axis, w,
                                                      radius);
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
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  fill_u8_kernel<<<(unsigned)blocks, 256, 0, s>>>(p, n, v);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace mb2
