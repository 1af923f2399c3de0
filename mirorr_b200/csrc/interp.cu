// interp.cu -- final-resampling interpolators for sm_100a: cubic B-spline and
// Welch-windowed sinc of radius 5, as GetInterpolatorFromString
// (itkMirorrPyramidImplement.txx:365-433) configures them for
// GetResampledImage (:436-479, a ResampleImageFilter with default value 0).
//
// Both map the output index idx to the input continuous index c = e + C idx
// (FP64, left to right, as the linear resampler) and write 0 outside
// -0.5 <= c < n - 0.5 (the interpolators' buffer test).  FP64 arithmetic is
// written with explicit round-to-nearest intrinsics (no contraction), so the
// B-spline results equal a plain C / numpy evaluation of the same expressions
// bit for bit; the sinc weights call sin(), so its results agree to rounding.
#include "kernels.cuh"

namespace mb2 {

namespace {

__device__ inline double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double dsub(double a, double b) { return __dsub_rn(a, b); }

__device__ inline void continuous_index(const ResampleMap &m, long long o, const int *on,
                                        double c[3]) {
  int i, j, k;
  split3(o, on[0], on[1], i, j, k);
  const double di = (double)i, dj = (double)j, dk = (double)k;
#pragma unroll
  for (int r = 0; r < 3; ++r)
    c[r] = dadd(dadd(dadd(m.e[r], dmul(m.C[3 * r], di)), dmul(m.C[3 * r + 1], dj)),
                dmul(m.C[3 * r + 2], dk));
}

// ---- cubic B-spline ---------------------------------------------------------
// Coefficients (the BSplineDecompositionImageFilter of order 3): along each
// axis in turn (x, y, z) every line c[0 .. N) of the FP64 coefficient volume
// is filtered in place with the single pole z = sqrt(3) - 2 (Unser's
// recursive B-spline prefilter):
//   c[n] *= lambda, lambda = (1 - z)(1 - 1/z);
//   c[0]  = causal initial value: with the horizon H = ceil(ln 1e-10 / ln|z|),
//           c[0] + sum_{n=1}^{H-1} z^n c[n] when H < N, otherwise the
//           mirror-symmetric full sum (z^(N-1) as a product of N-1 factors);
//   c[n] += z c[n-1]                     n = 1 .. N-1;
//   c[N-1] = z / (z^2 - 1) (z c[N-2] + c[N-1]);
//   c[n]  = z (c[n+1] - c[n])            n = N-2 .. 0.
// Lines of length 1 are left unchanged.
struct Pole {
  double z, lambda, iz, anti;  // pole, gain, 1/z, z / (z^2 - 1)
  int horizon;
};

__global__ void __launch_bounds__(256) bspline_line_kernel(double *coef, long long nlines,
                                                           int len, long long stride,
                                                           long long inner, long long outer_stride,
                                                           Pole pl) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nlines;
       l += (long long)gridDim.x * blockDim.x) {
    // line l: inner index l % inner (stride 1), outer index l / inner
    double *c = coef + (l % inner) + (l / inner) * outer_stride;
    if (len == 1) continue;
    const double z = pl.z;
    for (int n = 0; n < len; ++n) c[n * stride] = dmul(c[n * stride], pl.lambda);
    // causal initial value
    double zn = z;
    if (pl.horizon < len) {
      double sum = c[0];
      for (int n = 1; n < pl.horizon; ++n) {
        sum = dadd(sum, dmul(zn, c[n * stride]));
        zn = dmul(zn, z);
      }
      c[0] = sum;
    } else {
      double z2n = 1.0;
      for (int n = 0; n < len - 1; ++n) z2n = dmul(z2n, z);
      double sum = dadd(c[0], dmul(z2n, c[(long long)(len - 1) * stride]));
      z2n = dmul(z2n, dmul(z2n, pl.iz));
      for (int n = 1; n <= len - 2; ++n) {
        sum = dadd(sum, dmul(dadd(zn, z2n), c[n * stride]));
        zn = dmul(zn, z);
        z2n = dmul(z2n, pl.iz);
      }
      c[0] = __ddiv_rn(sum, dsub(1.0, dmul(zn, zn)));
    }
    for (int n = 1; n < len; ++n)
      c[n * stride] = dadd(c[n * stride], dmul(z, c[(n - 1) * stride]));
    const long long last = (long long)(len - 1) * stride;
    c[last] = dmul(pl.anti, dadd(dmul(z, c[last - stride]), c[last]));
    for (int n = len - 2; n >= 0; --n)
      c[n * stride] = dmul(z, dsub(c[(n + 1) * stride], c[n * stride]));
  }
}

__global__ void __launch_bounds__(256) to_double_kernel(const float *in, double *out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// Mirror boundary of the B-spline evaluation: index into [0, N) reflected at
// both ends (period 2N - 2), 0 for N = 1.
__device__ inline int mirror(int idx, int n) {
  if (n == 1) return 0;
  const int l2 = 2 * n - 2;
  idx = idx < 0 ? (-idx - l2 * ((-idx) / l2)) : (idx - l2 * (idx / l2));
  if (n <= idx) idx = l2 - idx;
  return idx;
}

// Evaluation (BSplineInterpolateImageFunction, order 3): per axis the support
// starts at floor(c) - 1; with w = c - floor(c) the weights are
//   w3 = w^3 / 6, w0 = 1/6 + w (w - 1) / 2 - w3, w2 = w + w0 - 2 w3,
//   w1 = 1 - w0 - w2 - w3;
// the 64 products ((wx wy) wz) coef are summed with x fastest.
__global__ void __launch_bounds__(256) bspline_eval_kernel(const double *coef, int nx, int ny,
                                                           int nz, ResampleMap m, int onx, int ony,
                                                           int onz, float *out) {
  const int on[3] = {onx, ony, onz}, nn[3] = {nx, ny, nz};
  const long long n = (long long)onx * ony * onz;
  const double sixth = 1.0 / 6.0;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    double c[3];
    continuous_index(m, o, on, c);
    bool inside = true;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (!(c[r] >= -0.5 && c[r] < (double)nn[r] - 0.5)) inside = false;
    if (!inside) {
      out[o] = 0.0f;
      continue;
    }
    double wt[3][4];
    int ix[3][4];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int b = (int)floor(c[r]);
      const double w = dsub(c[r], (double)b);
      const double w3 = dmul(dmul(dmul(sixth, w), w), w);
      const double w0 = dsub(dadd(sixth, dmul(dmul(0.5, w), dsub(w, 1.0))), w3);
      const double w2 = dsub(dadd(w, w0), dmul(2.0, w3));
      const double w1 = dsub(dsub(dsub(1.0, w0), w2), w3);
      wt[r][0] = w0; wt[r][1] = w1; wt[r][2] = w2; wt[r][3] = w3;
#pragma unroll
      for (int k = 0; k < 4; ++k) ix[r][k] = mirror(b - 1 + k, nn[r]);
    }
    double v = 0.0;
#pragma unroll
    for (int kz = 0; kz < 4; ++kz)
#pragma unroll
      for (int ky = 0; ky < 4; ++ky) {
        const long long row = ((long long)ix[2][kz] * ny + ix[1][ky]) * nx;
#pragma unroll
        for (int kx = 0; kx < 4; ++kx) {
          const double w = dmul(dmul(wt[0][kx], wt[1][ky]), wt[2][kz]);
          v = dadd(v, dmul(w, __ldg(coef + row + ix[0][kx])));
        }
      }
    out[o] = __double2float_rn(v);
  }
}

// ---- Welch-windowed sinc, radius 5 -------------------------------------------
// WindowedSincInterpolateImageFunction<R = 5, WelchWindowFunction> with the
// zero-flux Neumann (clamp-to-edge) boundary: per axis the base index is
// floor(c) and d = c - floor(c); the 2R taps at offsets 1-R .. R carry, for
// x = d + R - 1 - i (i = 0 .. 2R-1),
//   w(x) = (1 - x x / R^2) sin(pi x) / (pi x)   (1 at x = 0),
// or a delta at offset 0 when d = 0; the (2R)^3 products ((((p wx) wy) wz))
// are summed with x fastest.
constexpr int kSincR = 5;

__device__ inline double sinc_tap(double x) {
  const double welch = dsub(1.0, dmul(dmul(x, 1.0 / (kSincR * kSincR)), x));
  if (x == 0.0) return welch;
  const double px = dmul(3.14159265358979323846, x);
  return dmul(welch, __ddiv_rn(sin(px), px));
}

__global__ void __launch_bounds__(128) sinc_eval_kernel(const float *img, int nx, int ny, int nz,
                                                        ResampleMap m, int onx, int ony, int onz,
                                                        float *out) {
  constexpr int T = 2 * kSincR;
  const int on[3] = {onx, ony, onz}, nn[3] = {nx, ny, nz};
  const long long n = (long long)onx * ony * onz;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    double c[3];
    continuous_index(m, o, on, c);
    bool inside = true;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (!(c[r] >= -0.5 && c[r] < (double)nn[r] - 0.5)) inside = false;
    if (!inside) {
      out[o] = 0.0f;
      continue;
    }
    double wt[3][T];
    int ix[3][T];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int b = (int)floor(c[r]);
      const double d = dsub(c[r], (double)b);
      double x = dadd(d, (double)kSincR);
#pragma unroll
      for (int i = 0; i < T; ++i) {
        int q = b + i - (kSincR - 1);
        q = q < 0 ? 0 : (q > nn[r] - 1 ? nn[r] - 1 : q);
        ix[r][i] = q;
        if (d == 0.0) {
          wt[r][i] = i == kSincR - 1 ? 1.0 : 0.0;
        } else {
          x = dsub(x, 1.0);
          wt[r][i] = sinc_tap(x);
        }
      }
    }
    double v = 0.0;
    for (int kz = 0; kz < T; ++kz)
      for (int ky = 0; ky < T; ++ky) {
        const long long row = ((long long)ix[2][kz] * ny + ix[1][ky]) * nx;
#pragma unroll
        for (int kx = 0; kx < T; ++kx) {
          const double p = (double)__ldg(img + row + ix[0][kx]);
          v = dadd(v, dmul(dmul(dmul(p, wt[0][kx]), wt[1][ky]), wt[2][kz]));
        }
      }
    out[o] = __double2float_rn(v);
  }
}

long long grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return b > (long long)sm_count() * 64 ? (long long)sm_count() * 64 : (b < 1 ? 1 : b);
}

}  // namespace

mirorr_status launch_resample_bspline(const int in_size[3], const float *in, const int out_size[3],
                                      const ResampleMap &map, double *coef, float *out,
                                      cudaStream_t s) {
  const long long nin = (long long)in_size[0] * in_size[1] * in_size[2];
  const long long nout = (long long)out_size[0] * out_size[1] * out_size[2];
  if (nin <= 0 || nout <= 0) return MIRORR_OK;
  to_double_kernel<<<(unsigned)grid_for(nin, 256), 256, 0, s>>>(in, coef, nin);
  MB2_LAUNCH_CHECK();
  Pole pl;
  pl.z = sqrt(3.0) - 2.0;
  pl.lambda = (1.0 - pl.z) * (1.0 - 1.0 / pl.z);
  pl.iz = 1.0 / pl.z;
  pl.anti = pl.z / (pl.z * pl.z - 1.0);
  pl.horizon = (int)ceil(log(1e-10) / log(fabs(pl.z)));
  const long long nx = in_size[0], ny = in_size[1], nz = in_size[2];
  // x lines: inner 1, outer stride nx; y lines: inner nx, outer stride nx*ny;
  // z lines: inner nx*ny, outer stride 0 (one outer block)
  const long long lines[3] = {ny * nz, nx * nz, nx * ny};
  const long long stride[3] = {1, nx, nx * ny};
  const long long inner[3] = {1, nx, nx * ny};
  const long long ostride[3] = {nx, nx * ny, 0};
  for (int ax = 0; ax < 3; ++ax) {
    bspline_line_kernel<<<(unsigned)grid_for(lines[ax], 256), 256, 0, s>>>(
        coef, lines[ax], in_size[ax], stride[ax], inner[ax], ostride[ax], pl);
    MB2_LAUNCH_CHECK();
  }
  bspline_eval_kernel<<<(unsigned)grid_for(nout, 256), 256, 0, s>>>(
      coef, in_size[0], in_size[1], in_size[2], map, out_size[0], out_size[1], out_size[2], out);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

mirorr_status launch_resample_sinc(const int in_size[3], const float *in, const int out_size[3],
                                   const ResampleMap &map, float *out, cudaStream_t s) {
  const long long nout = (long long)out_size[0] * out_size[1] * out_size[2];
  if (nout <= 0) return MIRORR_OK;
  sinc_eval_kernel<<<(unsigned)grid_for(nout, 128), 128, 0, s>>>(
      in, in_size[0], in_size[1], in_size[2], map, out_size[0], out_size[1], out_size[2], out);
  MB2_LAUNCH_CHECK();
  return MIRORR_OK;
}

}  // namespace mb2
