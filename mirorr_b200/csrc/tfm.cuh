// tfm.cuh -- FP64 transform algebra for the registration path, usable on the
// host and on the device (the LTS solve runs in one device thread).
//
// It restates the semantics the reference relies on:
//   * itk::MatrixOffsetTransformBase: y = M (x - c) + c + t = M x + offset,
//     offset = t + c - M c; SetCenter/SetTranslation keep t and recompute the
//     offset; SetMatrix recomputes the offset then the matrix parameters;
//     Compose(other, pre) (pre: self(other(x)), else other(self(x))) keeps the
//     centre and recomputes the translation; GetInverse keeps the centre.
//   * itk::Euler3DTransform (ComputeZYX off): R = Rz Rx Ry, parameters
//     (ax, ay, az, tx, ty, tz); SetMatrix requires |M M^T - I| <= 1e-10 and
//     re-derives the matrix from the extracted angles.
//   * itk::AffineTransform: parameters = matrix row-major + translation.
//   * vnl_quaternion (x, y, z, r): rotation matrix, rotation_euler_angles
//     (R = Rz Ry Rx), axis(), angle(), (axis, angle) constructor.
//   * src/mirorr/vnl_utils.h: Denman-Beavers square root (:46-95) and
//     orthogonalize = U V^T of the SVD (:124-135).
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define MB2_HD __host__ __device__ inline
#else
#define MB2_HD inline
#endif

namespace mb2 {

enum { KIND_RIGID = 0, KIND_AFFINE = 1 };

// ---- small dense matrices (row-major) ------------------------------------
MB2_HD void m3_mul(const double *a, const double *b, double *o) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[3 * i + k] * b[3 * k + j];
      r[3 * i + j] = s;
    }
  for (int i = 0; i < 9; ++i) o[i] = r[i];
}
MB2_HD void m3_vec(const double *a, const double *v, double *o) {
  double r[3];
  for (int i = 0; i < 3; ++i) r[i] = a[3 * i] * v[0] + a[3 * i + 1] * v[1] + a[3 * i + 2] * v[2];
  o[0] = r[0]; o[1] = r[1]; o[2] = r[2];
}
MB2_HD void m3_transpose(const double *a, double *o) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[3 * j + i] = a[3 * i + j];
  for (int i = 0; i < 9; ++i) o[i] = r[i];
}
MB2_HD void m3_identity(double *o) {
  for (int i = 0; i < 9; ++i) o[i] = (i % 4 == 0) ? 1.0 : 0.0;
}
MB2_HD double m3_det(const double *a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// Gauss-Jordan inverse with partial pivoting; returns false when singular.
template <int N>
MB2_HD bool mn_inverse(const double *a, double *o) {
  double m[N][2 * N];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      m[i][j] = a[N * i + j];
      m[i][N + j] = (i == j) ? 1.0 : 0.0;
    }
  for (int c = 0; c < N; ++c) {
    int p = c;
    double best = fabs(m[c][c]);
    for (int r = c + 1; r < N; ++r)
      if (fabs(m[r][c]) > best) { best = fabs(m[r][c]); p = r; }
    if (best == 0.0) return false;
    if (p != c)
      for (int j = 0; j < 2 * N; ++j) { double t = m[c][j]; m[c][j] = m[p][j]; m[p][j] = t; }
    double inv = 1.0 / m[c][c];
    for (int j = 0; j < 2 * N; ++j) m[c][j] *= inv;
    for (int r = 0; r < N; ++r) {
      if (r == c) continue;
      double f = m[r][c];
      if (f != 0.0)
        for (int j = 0; j < 2 * N; ++j) m[r][j] -= f * m[c][j];
    }
  }
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) o[N * i + j] = m[i][N + j];
  return true;
}

template <int N>
MB2_HD void mn_mul(const double *a, const double *b, double *o) {
  double r[N * N];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0.0;
      for (int k = 0; k < N; ++k) s += a[N * i + k] * b[N * k + j];
      r[N * i + j] = s;
    }
  for (int i = 0; i < N * N; ++i) o[i] = r[i];
}

// Cyclic Jacobi eigen-decomposition of a symmetric NxN matrix.  On return
// w[] holds eigenvalues in ascending order and column k of v is the
// eigenvector of w[k].
template <int N>
MB2_HD void jacobi_eigen(const double *a_in, double *w, double *v) {
  double a[N * N];
  for (int i = 0; i < N * N; ++i) a[i] = a_in[i];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) v[N * i + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < N; ++i) {
      diag += a[N * i + i] * a[N * i + i];
      for (int j = i + 1; j < N; ++j) off += a[N * i + j] * a[N * i + j];
    }
    if (off <= 1e-32 * diag || off == 0.0) break;
    for (int p = 0; p < N; ++p)
      for (int q = p + 1; q < N; ++q) {
        double apq = a[N * p + q];
        if (apq == 0.0) continue;
        double app = a[N * p + p], aqq = a[N * q + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < N; ++k) {
          double akp = a[N * k + p], akq = a[N * k + q];
          a[N * k + p] = c * akp - s * akq;
          a[N * k + q] = s * akp + c * akq;
        }
        for (int k = 0; k < N; ++k) {
          double apk = a[N * p + k], aqk = a[N * q + k];
          a[N * p + k] = c * apk - s * aqk;
          a[N * q + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < N; ++k) {
          double vkp = v[N * k + p], vkq = v[N * k + q];
          v[N * k + p] = c * vkp - s * vkq;
          v[N * k + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < N; ++i) w[i] = a[N * i + i];
  // sort ascending (selection sort on columns)
  for (int i = 0; i < N; ++i) {
    int m = i;
    for (int j = i + 1; j < N; ++j)
      if (w[j] < w[m]) m = j;
    if (m != i) {
      double t = w[i]; w[i] = w[m]; w[m] = t;
      for (int k = 0; k < N; ++k) { double u = v[N * k + i]; v[N * k + i] = v[N * k + m]; v[N * k + m] = u; }
    }
  }
}

// Orthogonal polar factor U V^T of a (non-singular) 3x3 matrix:
// M (M^T M)^(-1/2), computed from the eigen-decomposition of M^T M.
MB2_HD void orthogonalize3(const double *m, double *o) {
  double mt[9], mtm[9], w[3], v[9];
  m3_transpose(m, mt);
  m3_mul(mt, m, mtm);
  jacobi_eigen<3>(mtm, w, v);
  double isq[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) {
        double lk = w[k] > 0.0 ? 1.0 / sqrt(w[k]) : 0.0;
        s += v[3 * i + k] * lk * v[3 * j + k];
      }
      isq[3 * i + j] = s;
    }
  m3_mul(m, isq, o);
}

// Inverse of a homogeneous affine 4x4 matrix [A t; 0 0 0 1] (row-major):
// [A^-1, -A^-1 t; 0 0 0 1], with A^-1 from its cofactors.  False when A is
// singular.
MB2_HD bool affine4_inverse(const double *m, double *o) {
  const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6];
  const double g = m[8], h = m[9], k = m[10];
  const double c00 = e * k - f * h, c01 = f * g - d * k, c02 = d * h - e * g;
  const double det = a * c00 + b * c01 + c * c02;
  if (det == 0.0) return false;
  const double r = 1.0 / det;
  double ia[9];
  ia[0] = c00 * r; ia[1] = (c * h - b * k) * r; ia[2] = (b * f - c * e) * r;
  ia[3] = c01 * r; ia[4] = (a * k - c * g) * r; ia[5] = (c * d - a * f) * r;
  ia[6] = c02 * r; ia[7] = (b * g - a * h) * r; ia[8] = (a * e - b * d) * r;
  for (int i = 0; i < 3; ++i) {
    o[4 * i + 0] = ia[3 * i + 0];
    o[4 * i + 1] = ia[3 * i + 1];
    o[4 * i + 2] = ia[3 * i + 2];
    o[4 * i + 3] = -(ia[3 * i + 0] * m[3] + ia[3 * i + 1] * m[7] + ia[3 * i + 2] * m[11]);
  }
  o[12] = 0.0; o[13] = 0.0; o[14] = 0.0; o[15] = 1.0;
  return true;
}

// Denman-Beavers square root of a homogeneous affine 4x4 matrix
// (vnl_utils.h:46-95) with EPS = 1e-14, MAX_ITER = 50 as called from
// itkSymMirorrRegistrationMethod.txx.  Every iterate keeps the last row
// 0 0 0 1, so the inverses are the affine ones.
MB2_HD void matrix_sqrt4(const double *m, double *y_out) {
  double y[16], z[16], iy[16], iz[16], d[16];
  for (int i = 0; i < 16; ++i) { y[i] = m[i]; z[i] = (i % 5 == 0) ? 1.0 : 0.0; }
  double dd = 1.7976931348623157e308;
  int it = 0;
  while (dd > 1e-14 && it < 50) {
    affine4_inverse(z, iz);
    affine4_inverse(y, iy);
    for (int i = 0; i < 16; ++i) {
      const double ny = 0.5 * (y[i] + iz[i]), nz = 0.5 * (z[i] + iy[i]);
      y[i] = ny;
      z[i] = nz;
    }
    ++it;
    mn_mul<4>(y, y, d);
    dd = 0.0;
    for (int i = 0; i < 16; ++i) {
      double a = fabs(d[i] - m[i]);
      if (a > dd) dd = a;
    }
  }
  for (int i = 0; i < 16; ++i) y_out[i] = y[i];
}

// ---- Euler3D (Z*X*Y) -------------------------------------------------------
MB2_HD void euler_zxy_matrix(const double *ang, double *o) {
  double cx = cos(ang[0]), sx = sin(ang[0]);
  double cy = cos(ang[1]), sy = sin(ang[1]);
  double cz = cos(ang[2]), sz = sin(ang[2]);
  double rx[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
  double ry[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
  double rz[9] = {cz, -sz, 0, sz, cz, 0, 0, 0, 1};
  double t[9];
  m3_mul(rz, rx, t);
  m3_mul(t, ry, o);
}

MB2_HD void euler_zxy_angles(const double *m, double *ang) {
  double s = m[7];
  if (s > 1.0) s = 1.0;
  if (s < -1.0) s = -1.0;
  ang[0] = asin(s);
  double a = cos(ang[0]);
  if (fabs(a) > 0.00005) {
    ang[1] = atan2(-m[6] / a, m[8] / a);
    ang[2] = atan2(-m[1] / a, m[4] / a);
  } else {
    ang[2] = 0.0;
    ang[1] = atan2(m[3], m[0]);
  }
}

// ---- transform -------------------------------------------------------------
struct Tfm {
  int kind;
  double M[9];
  double off[3];
  double c[3];
  double t[3];
  double ang[3];
};

MB2_HD void tfm_identity(Tfm &a, int kind) {
  a.kind = kind;
  m3_identity(a.M);
  for (int i = 0; i < 3; ++i) { a.off[i] = 0; a.c[i] = 0; a.t[i] = 0; a.ang[i] = 0; }
}
MB2_HD void tfm_compute_offset(Tfm &a) {
  double mc[3];
  m3_vec(a.M, a.c, mc);
  for (int i = 0; i < 3; ++i) a.off[i] = a.t[i] + a.c[i] - mc[i];
}
MB2_HD void tfm_compute_translation(Tfm &a) {
  double mc[3];
  m3_vec(a.M, a.c, mc);
  for (int i = 0; i < 3; ++i) a.t[i] = a.off[i] - a.c[i] + mc[i];
}
MB2_HD void tfm_compute_matrix_params(Tfm &a) {
  if (a.kind == KIND_RIGID) {
    euler_zxy_angles(a.M, a.ang);
    euler_zxy_matrix(a.ang, a.M);
  }
}
MB2_HD void tfm_set_center(Tfm &a, const double *c) {
  for (int i = 0; i < 3; ++i) a.c[i] = c[i];
  tfm_compute_offset(a);
}
MB2_HD void tfm_set_translation(Tfm &a, const double *t) {
  for (int i = 0; i < 3; ++i) a.t[i] = t[i];
  tfm_compute_offset(a);
}
// Returns false (and leaves the transform unchanged) when a rigid transform is
// given a matrix that is not orthogonal within 1e-10.
MB2_HD bool tfm_set_matrix(Tfm &a, const double *m) {
  if (a.kind == KIND_RIGID) {
    double mt[9], p[9];
    m3_transpose(m, mt);
    m3_mul(m, mt, p);
    for (int i = 0; i < 9; ++i) {
      double d = p[i] - ((i % 4 == 0) ? 1.0 : 0.0);
      if (fabs(d) > 1e-10) return false;
    }
  }
  for (int i = 0; i < 9; ++i) a.M[i] = m[i];
  tfm_compute_offset(a);
  tfm_compute_matrix_params(a);
  return true;
}
MB2_HD int tfm_nparams(const Tfm &a) { return a.kind == KIND_RIGID ? 6 : 12; }
MB2_HD void tfm_params(const Tfm &a, double *p) {
  if (a.kind == KIND_RIGID) {
    for (int i = 0; i < 3; ++i) { p[i] = a.ang[i]; p[3 + i] = a.t[i]; }
  } else {
    for (int i = 0; i < 9; ++i) p[i] = a.M[i];
    for (int i = 0; i < 3; ++i) p[9 + i] = a.t[i];
  }
}
MB2_HD void tfm_set_params(Tfm &a, const double *p) {
  if (a.kind == KIND_RIGID) {
    for (int i = 0; i < 3; ++i) { a.ang[i] = p[i]; a.t[i] = p[3 + i]; }
    euler_zxy_matrix(a.ang, a.M);
  } else {
    for (int i = 0; i < 9; ++i) a.M[i] = p[i];
    for (int i = 0; i < 3; ++i) a.t[i] = p[9 + i];
  }
  tfm_compute_offset(a);
}
MB2_HD void tfm_compose(Tfm &a, const Tfm &o, bool pre) {
  double nm[9], noff[3];
  if (pre) {
    m3_vec(a.M, o.off, noff);
    for (int i = 0; i < 3; ++i) noff[i] += a.off[i];
    m3_mul(a.M, o.M, nm);
  } else {
    m3_vec(o.M, a.off, noff);
    for (int i = 0; i < 3; ++i) noff[i] += o.off[i];
    m3_mul(o.M, a.M, nm);
  }
  for (int i = 0; i < 9; ++i) a.M[i] = nm[i];
  for (int i = 0; i < 3; ++i) a.off[i] = noff[i];
  tfm_compute_translation(a);
  tfm_compute_matrix_params(a);
}
MB2_HD bool tfm_inverse(const Tfm &a, Tfm &o) {
  double mi[9];
  if (!mn_inverse<3>(a.M, mi)) return false;
  o.kind = a.kind;
  for (int i = 0; i < 3; ++i) { o.c[i] = a.c[i]; o.ang[i] = 0; }
  for (int i = 0; i < 9; ++i) o.M[i] = mi[i];
  double v[3];
  m3_vec(mi, a.off, v);
  for (int i = 0; i < 3; ++i) o.off[i] = -v[i];
  tfm_compute_translation(o);
  tfm_compute_matrix_params(o);
  return true;
}
MB2_HD void tfm_apply(const Tfm &a, const double *x, double *y) {
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int j = 0; j < 3; ++j) s += a.M[3 * i + j] * x[j];
    y[i] = s + a.off[i];
  }
}
// itkTransformUtils.h:22-35
MB2_HD void tfm_center_to_origin(Tfm &a) {
  double off[3] = {a.off[0], a.off[1], a.off[2]};
  double z[3] = {0, 0, 0};
  tfm_set_center(a, z);
  tfm_set_translation(a, off);
}
// itkTransformUtils.h:42-57
MB2_HD void tfm_update_center(Tfm &a, const double *c2) {
  tfm_center_to_origin(a);
  double ic[3] = {-c2[0], -c2[1], -c2[2]};
  tfm_set_center(a, ic);
  double off[3] = {a.off[0], a.off[1], a.off[2]};
  tfm_set_center(a, c2);
  tfm_set_translation(a, off);
}

// ---- vnl_quaternion (x, y, z, r) --------------------------------------------
MB2_HD void quat_rotation(const double *q, double *r) {
  double x = q[0], y = q[1], z = q[2], w = q[3];
  double rt[9];
  double x2 = x * x, y2 = y * y, z2 = z * z, r2 = w * w;
  double xy = x * y, yz = y * z, zx = z * x, rx = w * x, ry = w * y, rz = w * z;
  rt[0] = r2 + x2 - y2 - z2;
  rt[4] = r2 - x2 + y2 - z2;
  rt[8] = r2 - x2 - y2 + z2;
  rt[1] = 2 * (xy + rz);
  rt[2] = 2 * (zx - ry);
  rt[5] = 2 * (yz + rx);
  rt[3] = 2 * (xy - rz);
  rt[6] = 2 * (zx + ry);
  rt[7] = 2 * (yz - rx);
  m3_transpose(rt, r);
}
MB2_HD void quat_euler_angles(const double *q, double *ang) {
  double r[9], rt[9];
  quat_rotation(q, r);
  m3_transpose(r, rt);
  double xy = sqrt(rt[0] * rt[0] + rt[1] * rt[1]);
  if (xy > 2.220446049250313e-16 * 8.0) {
    ang[0] = atan2(rt[5], rt[8]);
    ang[1] = atan2(-rt[2], xy);
    ang[2] = atan2(rt[1], rt[0]);
  } else {
    ang[0] = atan2(-rt[7], rt[4]);
    ang[1] = atan2(-rt[2], xy);
    ang[2] = 0.0;
  }
}
MB2_HD void quat_axis_angle(const double *q, double *axis, double *angle) {
  double mag = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  *angle = 2.0 * atan2(mag, q[3]);
  if (mag == 0.0) { axis[0] = 0; axis[1] = 0; axis[2] = 1; }
  else { axis[0] = q[0] / mag; axis[1] = q[1] / mag; axis[2] = q[2] / mag; }
}
MB2_HD void quat_from_axis_angle(const double *axis, double angle, double *q) {
  double a = angle * 0.5, s = sin(a);
  q[0] = s * axis[0]; q[1] = s * axis[1]; q[2] = s * axis[2]; q[3] = cos(a);
}

// Horn's quaternion from the moments of centred point pairs.  Z is the 6x6
// second-moment matrix of z = (a0,a1,a2,b0,b1,b2) with a = initial - mean,
// b = moved - mean.  The per-point matrix Q of CalculateRigidQuaternion
// (itkMirorrRegistrationMethod.txx:1063-1106) is linear in z, so
// sum Q^T Q = sum_i C_i^T Z C_i over its coefficient vectors.  Returns the
// eigenvector of the smallest eigenvalue as (x, y, z, r).
MB2_HD void horn_quaternion(const double *Z, double *q) {
  // tot = sum over the subset of Q^T Q, Q the 4x4 matrix of one pair whose
  // entries are +-1 times the six centred coordinates z_k: entry (j, l) is
  // sum_i sum_{a,b} c(i,j,a) c(i,l,b) Z[a][b] over the non-zero coefficients
  // c (all +-1), written out term by term in that order (i, then a, then b),
  // so every entry is the same sequence of additions as the coefficient form
  double tot[16];
  {  // entry (0, 0)
    double s = 0.0;
    s += Z[0]; s -= Z[3]; s -= Z[18]; s += Z[21]; s += Z[7]; s -= Z[10]; s -= Z[25]; s += Z[28];
    s += Z[14]; s -= Z[17]; s -= Z[32]; s += Z[35];
    tot[0] = s;
  }
  {  // entry (0, 1)
    double s = 0.0;
    s -= Z[8]; s -= Z[11]; s += Z[26]; s += Z[29]; s += Z[13]; s += Z[16]; s -= Z[31];
    s -= Z[34];
    tot[1] = s;
  }
  {  // entry (0, 2)
    double s = 0.0;
    s += Z[2]; s += Z[5]; s -= Z[20]; s -= Z[23]; s -= Z[12]; s -= Z[15]; s += Z[30];
    s += Z[33];
    tot[2] = s;
  }
  {  // entry (0, 3)
    double s = 0.0;
    s -= Z[1]; s -= Z[4]; s += Z[19]; s += Z[22]; s += Z[6]; s += Z[9]; s -= Z[24]; s -= Z[27];
    tot[3] = s;
  }
  {  // entry (1, 0)
    double s = 0.0;
    s -= Z[13]; s += Z[16]; s -= Z[31]; s += Z[34]; s += Z[8]; s -= Z[11]; s += Z[26];
    s -= Z[29];
    tot[4] = s;
  }
  {  // entry (1, 1)
    double s = 0.0;
    s += Z[0]; s -= Z[3]; s -= Z[18]; s += Z[21]; s += Z[14]; s += Z[17]; s += Z[32];
    s += Z[35]; s += Z[7]; s += Z[10]; s += Z[25]; s += Z[28];
    tot[5] = s;
  }
  {  // entry (1, 2)
    double s = 0.0;
    s += Z[1]; s -= Z[4]; s -= Z[19]; s += Z[22]; s -= Z[6]; s -= Z[9]; s -= Z[24]; s -= Z[27];
    tot[6] = s;
  }
  {  // entry (1, 3)
    double s = 0.0;
    s += Z[2]; s -= Z[5]; s -= Z[20]; s += Z[23]; s -= Z[12]; s -= Z[15]; s -= Z[30];
    s -= Z[33];
    tot[7] = s;
  }
  {  // entry (2, 0)
    double s = 0.0;
    s += Z[12]; s -= Z[15]; s += Z[30]; s -= Z[33]; s -= Z[2]; s += Z[5]; s -= Z[20];
    s += Z[23];
    tot[8] = s;
  }
  {  // entry (2, 1)
    double s = 0.0;
    s += Z[6]; s -= Z[9]; s -= Z[24]; s += Z[27]; s -= Z[1]; s -= Z[4]; s -= Z[19]; s -= Z[22];
    tot[9] = s;
  }
  {  // entry (2, 2)
    double s = 0.0;
    s += Z[7]; s -= Z[10]; s -= Z[25]; s += Z[28]; s += Z[14]; s += Z[17]; s += Z[32];
    s += Z[35]; s += Z[0]; s += Z[3]; s += Z[18]; s += Z[21];
    tot[10] = s;
  }
  {  // entry (2, 3)
    double s = 0.0;
    s += Z[8]; s -= Z[11]; s -= Z[26]; s += Z[29]; s -= Z[13]; s -= Z[16]; s -= Z[31];
    s -= Z[34];
    tot[11] = s;
  }
  {  // entry (3, 0)
    double s = 0.0;
    s -= Z[6]; s += Z[9]; s -= Z[24]; s += Z[27]; s += Z[1]; s -= Z[4]; s += Z[19]; s -= Z[22];
    tot[12] = s;
  }
  {  // entry (3, 1)
    double s = 0.0;
    s += Z[12]; s -= Z[15]; s -= Z[30]; s += Z[33]; s -= Z[2]; s -= Z[5]; s -= Z[20];
    s -= Z[23];
    tot[13] = s;
  }
  {  // entry (3, 2)
    double s = 0.0;
    s += Z[13]; s -= Z[16]; s -= Z[31]; s += Z[34]; s -= Z[8]; s -= Z[11]; s -= Z[26];
    s -= Z[29];
    tot[14] = s;
  }
  {  // entry (3, 3)
    double s = 0.0;
    s += Z[14]; s -= Z[17]; s -= Z[32]; s += Z[35]; s += Z[7]; s += Z[10]; s += Z[25];
    s += Z[28]; s += Z[0]; s += Z[3]; s += Z[18]; s += Z[21];
    tot[15] = s;
  }
  double ev[4], vec[16];
  jacobi_eigen<4>(tot, ev, vec);
  q[0] = vec[4 * 1 + 0];
  q[1] = vec[4 * 2 + 0];
  q[2] = vec[4 * 3 + 0];
  q[3] = vec[4 * 0 + 0];
}

// ---- LTS steps ---------------------------------------------------------------
// Moments of the LTS subset of one inner iteration.
struct LtsMoments {
  double n;         // subset size
  double mean_i[3]; // barycentre of initial points
  double mean_m[3]; // barycentre of moved points
  double Z[36];     // second moments of (initial - mean_i, moved - mean_m), summed
};

// Working state of one LTS fit (one OptimizeTransform call).
struct LtsState {
  int kind;
  int symmetric;
  double lts_keep;
  Tfm tfm;        // m_Transform
  Tfm t12f, t12b; // half-space transforms (symmetric)
  Tfm fin;        // final_transform (classic) / final_transformF (symmetric)
  Tfm finb;       // final_transformB (symmetric)
  double rc[3];
  double last_params[12];
  double fraction;
  double delta, last_delta;
  int iter;       // completed inner iterations
  int running;    // 1 while the while-condition holds
  int failed;
};

MB2_HD bool lts_continue(const LtsState &s) {
  return s.delta > 1e-3 && (s.iter - 1) < 100 && fabs(s.delta - s.last_delta) > 1e-3;
}

MB2_HD void lts_begin(LtsState &s) {
  for (int i = 0; i < 3; ++i) s.rc[i] = s.tfm.c[i];
  tfm_identity(s.fin, s.kind);
  tfm_set_center(s.fin, s.rc);
  tfm_identity(s.finb, s.kind);
  tfm_set_center(s.finb, s.rc);
  tfm_params(s.fin, s.last_params);
  s.fraction = 1.0;
  s.last_delta = 0.0;
  s.delta = 1.0;
  s.iter = 0;
  s.running = 1;
  s.failed = 0;
}

MB2_HD void cov_from_Z(const double *Z, int ra, int cb, double n, double *o) {
  // o[r][c] = sum A[r] * B[c] / n with A = z[ra..ra+2], B = z[cb..cb+2]
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o[3 * r + c] = Z[6 * (ra + r) + (cb + c)] / n;
}

// Least-squares affine A = Cov(y, x) Cov(x, x)^-1, skipping the inverse when
// |det Cov(x, x)| < 1e-4 (itkMirorrRegistrationMethod.txx:871-883).
MB2_HD void affine_ls(const double *Z, int xo, int yo, double n, double *rot) {
  double oxy[9], oxx[9];
  cov_from_Z(Z, yo, xo, n, oxy);
  cov_from_Z(Z, xo, xo, n, oxx);
  for (int i = 0; i < 9; ++i) rot[i] = oxy[i];
  if (fabs(m3_det(oxx)) >= 1e-4) {
    double inv[9];
    if (mn_inverse<3>(oxx, inv)) m3_mul(oxy, inv, rot);
  }
}

// One inner iteration of the classic fit, after the subset moments are known
// (itkMirorrRegistrationMethod.txx:841-998).
MB2_HD void lts_classic_step(LtsState &s, const LtsMoments &mo) {
  double np[12];
  for (int i = 0; i < 12; ++i) np[i] = s.last_params[i];
  const double *im = mo.mean_i, *mm = mo.mean_m;
  double mfc[3], ifc[3];
  for (int i = 0; i < 3; ++i) { mfc[i] = mm[i] - s.rc[i]; ifc[i] = im[i] - s.rc[i]; }
  double rot[9];
  if (s.kind == KIND_AFFINE) {
    affine_ls(mo.Z, 0, 3, mo.n, rot);
    double ri[3];
    m3_vec(rot, ifc, ri);
    for (int i = 0; i < 9; ++i) np[i] = rot[i];
    for (int i = 0; i < 3; ++i) np[9 + i] = mfc[i] - ri[i];
  } else {
    double q[4];
    horn_quaternion(mo.Z, q);
    quat_rotation(q, rot);
    double ri[3], ang[3];
    m3_vec(rot, ifc, ri);
    quat_euler_angles(q, ang);
    for (int i = 0; i < 3; ++i) { np[i] = ang[i]; np[3 + i] = mfc[i] - ri[i]; }
  }
  s.last_delta = s.delta;
  double d = 0.0;
  int npar = tfm_nparams(s.fin);
  for (int i = 0; i < npar; ++i) { double e = s.last_params[i] - np[i]; d += e * e; }
  s.delta = d;
  for (int i = 0; i < 3; ++i) s.rc[i] = im[i];
  tfm_set_center(s.fin, s.rc);
  tfm_set_params(s.fin, np);
}

MB2_HD void half_step(const double *K, const double *trans, double *m12) {
  double m[16];
  for (int i = 0; i < 16; ++i) m[i] = 0.0;
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) m[4 * r + c] = K[3 * r + c];
    m[4 * r + 3] = trans[r];
  }
  m[15] = 1.0;
  matrix_sqrt4(m, m12);
}

// One inner iteration of the symmetric fit (itkSymMirorrRegistrationMethod.txx:865-1432)
// in three parts: lts_symmetric_pre (the two least-squares fits and the
// averaged half-way matrices Kf, Kb with translations tf, tb), the two
// independent square roots half_step(Kf, tf) and half_step(Kb, tb), which the
// device runs on two lanes at once, and lts_symmetric_post.
struct SymHalf {
  double np[12];
  double K[2][9];
  double t[2][3];
};

MB2_HD void lts_symmetric_pre(LtsState &s, const LtsMoments &mo, SymHalf &h) {
  double *np = h.np;
  for (int i = 0; i < 12; ++i) np[i] = s.last_params[i];
  const double *im = mo.mean_i, *mm = mo.mean_m;
  double translation[3], ntrans[3];
  for (int i = 0; i < 3; ++i) { translation[i] = mm[i] - im[i]; ntrans[i] = -translation[i]; }
  Tfm &ff = s.fin;
  Tfm &fb = s.finb;
  if (s.kind == KIND_AFFINE) {
    double rf[9], rb[9];
    affine_ls(mo.Z, 0, 3, mo.n, rf);
    affine_ls(mo.Z, 3, 0, mo.n, rb);
    for (int i = 0; i < 9; ++i) np[i] = rf[i];
    for (int i = 0; i < 3; ++i) np[9 + i] = translation[i];
    double pf[12], pb[12];
    for (int i = 0; i < 9; ++i) { pf[i] = rf[i]; pb[i] = rb[i]; }
    for (int i = 0; i < 3; ++i) { pf[9 + i] = translation[i]; pb[9 + i] = ntrans[i]; }
    tfm_set_center(ff, im); tfm_set_params(ff, pf);
    tfm_set_center(fb, mm); tfm_set_params(fb, pb);
    double ibm[9], ifm[9], K[9], Mb[9];
    mn_inverse<3>(fb.M, ibm);
    mn_inverse<3>(ff.M, ifm);
    for (int i = 0; i < 9; ++i) { K[i] = (ff.M[i] + ibm[i]) / 2.0; Mb[i] = (ifm[i] + fb.M[i]) / 2.0; }
    tfm_set_matrix(ff, K);
    tfm_set_matrix(fb, Mb);
  } else {
    double q[4], ang[3], axis[3], angle, qf[4], qb[4], af[3], ab[3];
    horn_quaternion(mo.Z, q);
    quat_euler_angles(q, ang);
    quat_axis_angle(q, axis, &angle);
    quat_from_axis_angle(axis, angle, qf);
    quat_from_axis_angle(axis, -angle, qb);
    quat_euler_angles(qf, af);
    quat_euler_angles(qb, ab);
    for (int i = 0; i < 3; ++i) { np[i] = ang[i]; np[3 + i] = translation[i]; }
    double pf[6] = {af[0], af[1], af[2], translation[0], translation[1], translation[2]};
    double pb[6] = {ab[0], ab[1], ab[2], ntrans[0], ntrans[1], ntrans[2]};
    tfm_set_center(ff, im); tfm_set_params(ff, pf);
    tfm_set_center(fb, mm); tfm_set_params(fb, pb);
    double ibm[9], K[9], Ko[9], Kt[9];
    mn_inverse<3>(fb.M, ibm);
    for (int i = 0; i < 9; ++i) K[i] = (ff.M[i] + ibm[i]) / 2.0;
    orthogonalize3(K, Ko);
    m3_transpose(Ko, Kt);
    if (!tfm_set_matrix(ff, Ko) || !tfm_set_matrix(fb, Kt)) s.failed = 1;
  }
  double offf[3] = {ff.off[0], ff.off[1], ff.off[2]};
  double offb[3] = {fb.off[0], fb.off[1], fb.off[2]};
  double zero[3] = {0, 0, 0};
  tfm_set_center(ff, zero); tfm_set_center(fb, zero);
  tfm_set_translation(ff, offf); tfm_set_translation(fb, offb);
  Tfm iF, iB;
  tfm_inverse(ff, iF);
  tfm_inverse(fb, iB);
  double Kf[9], Kb[9], tf[3], tb[3];
  for (int i = 0; i < 9; ++i) { Kf[i] = (ff.M[i] + iB.M[i]) / 2.0; Kb[i] = (iF.M[i] + fb.M[i]) / 2.0; }
  if (s.kind == KIND_RIGID) {
    double a[9], b[9];
    orthogonalize3(Kf, a); orthogonalize3(Kb, b);
    for (int i = 0; i < 9; ++i) { Kf[i] = a[i]; Kb[i] = b[i]; }
  }
  for (int i = 0; i < 3; ++i) { tf[i] = (ff.t[i] + iB.t[i]) / 2.0; tb[i] = (iF.t[i] + fb.t[i]) / 2.0; }
  for (int i = 0; i < 9; ++i) { h.K[0][i] = Kf[i]; h.K[1][i] = Kb[i]; }
  for (int i = 0; i < 3; ++i) { h.t[0][i] = tf[i]; h.t[1][i] = tb[i]; }
}

MB2_HD void lts_symmetric_post(LtsState &s, const SymHalf &h, const double *m12,
                               const double *im12) {
  const double *np = h.np;
  Tfm &ff = s.fin;
  Tfm &fb = s.finb;
  double k3[9], l3[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) { k3[3 * r + c] = m12[4 * r + c]; l3[3 * r + c] = im12[4 * r + c]; }
  Tfm ffs = ff, fbs = fb;
  if (!tfm_set_matrix(ff, k3) || !tfm_set_matrix(fb, l3)) {
    // SymMirorrRegistrationMethod re-orthogonalises both on rejection (:1327-1342)
    ff = ffs; fb = fbs;
    double ko[9], lo[9];
    orthogonalize3(k3, ko);
    orthogonalize3(l3, lo);
    tfm_set_matrix(ff, ko);
    tfm_set_matrix(fb, lo);
  }
  double t12[3] = {m12[3], m12[7], m12[11]}, it12[3] = {im12[3], im12[7], im12[11]};
  tfm_set_translation(ff, t12);
  tfm_set_translation(fb, it12);
  s.last_delta = s.delta;
  double d = 0.0;
  int npar = tfm_nparams(s.tfm);
  for (int i = 0; i < npar; ++i) { double e = s.last_params[i] - np[i]; d += e * e; }
  s.delta = d;
  for (int i = 0; i < 12; ++i) s.last_params[i] = np[i];
}

MB2_HD void lts_symmetric_step(LtsState &s, const LtsMoments &mo) {
  SymHalf h;
  lts_symmetric_pre(s, mo, h);
  double m12[16], im12[16];
  half_step(h.K[0], h.t[0], m12);
  half_step(h.K[1], h.t[1], im12);
  lts_symmetric_post(s, h, m12, im12);
}

// After the inner loop: m_Transform->Compose(final, true) (classic) or the
// half-space composition (symmetric, itkSymMirorrRegistrationMethod.txx:1452-1462).
MB2_HD void lts_finish(LtsState &s) {
  if (!s.symmetric) {
    tfm_compose(s.tfm, s.fin, true);
  } else {
    tfm_compose(s.t12f, s.fin, true);
    tfm_compose(s.t12b, s.finb, true);
    Tfm ib;
    tfm_inverse(s.t12b, ib);
    tfm_identity(s.tfm, s.tfm.kind);
    tfm_compose(s.tfm, ib, true);
    tfm_compose(s.tfm, s.t12f, false);
  }
}

// ComputeHalfSpaceTransforms (itkSymMirorrRegistrationMethod.txx:139-201).
MB2_HD void half_space(const Tfm &t, Tfm &f, Tfm &b) {
  double m[16], mi[16], m12[16], im12[16];
  for (int i = 0; i < 16; ++i) m[i] = 0.0;
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) m[4 * r + c] = t.M[3 * r + c];
    m[4 * r + 3] = t.t[r];
  }
  m[15] = 1.0;
  matrix_sqrt4(m, m12);
  affine4_inverse(m, mi);
  matrix_sqrt4(mi, im12);
  tfm_identity(f, t.kind);
  tfm_identity(b, t.kind);
  double k3[9], l3[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) { k3[3 * r + c] = m12[4 * r + c]; l3[3 * r + c] = im12[4 * r + c]; }
  if (!tfm_set_matrix(f, k3)) { double o[9]; orthogonalize3(k3, o); tfm_set_matrix(f, o); }
  if (!tfm_set_matrix(b, l3)) { double o[9]; orthogonalize3(l3, o); tfm_set_matrix(b, o); }
  double tf[3] = {m12[3], m12[7], m12[11]}, tb[3] = {im12[3], im12[7], im12[11]};
  tfm_set_translation(f, tf);
  tfm_set_translation(b, tb);
}

}  // namespace mb2
