"""Host-side checks of the transform algebra shared by the device code
(mirorr_b200/csrc/tfm.cuh compiled as plain C++, no GPU).

The rigid LTS fit's Horn matrix (sum of Q^T Q over the subset, Q the 4x4
quaternion matrix of a point pair, itkMirorrRegistrationMethod.txx:1063-1106)
is written out term by term in tfm.cuh.  Its coefficients are all +-1, so
every entry is a plain sequence of additions; this test rebuilds the matrix
from the coefficient table in the table's summation order (i, then a, then
b) and requires the quaternions to be bit-identical on random inputs,
including zeros, tiny and large values.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r'''
#include <cstdio>
#include <cstring>
#include <random>
#include <initializer_list>
#include "tfm.cuh"

// The coefficient-table form: Q[i][j] = sum_k coef(i, j, k) z_k.
static void horn_table(const double *Z, double *q) {
  double coef[16 * 6];
  for (double &c : coef) c = 0.0;
  auto set = [&](int i, int j, int k, double v) { coef[(i * 4 + j) * 6 + k] = v; };
  set(0, 1, 0, 1.0); set(0, 1, 3, -1.0);
  set(0, 2, 1, 1.0); set(0, 2, 4, -1.0);
  set(0, 3, 2, 1.0); set(0, 3, 5, -1.0);
  set(1, 2, 2, -1.0); set(1, 2, 5, -1.0);
  set(1, 3, 1, 1.0); set(1, 3, 4, 1.0);
  set(2, 3, 0, -1.0); set(2, 3, 3, -1.0);
  for (int i = 0; i < 4; ++i)
    for (int j = i + 1; j < 4; ++j)
      for (int k = 0; k < 6; ++k) coef[(j * 4 + i) * 6 + k] = -coef[(i * 4 + j) * 6 + k];
  double tot[16];
  for (int j = 0; j < 4; ++j)
    for (int l = 0; l < 4; ++l) {
      double s = 0.0;
      for (int i = 0; i < 4; ++i) {
        const double *u = &coef[(i * 4 + j) * 6];
        const double *w = &coef[(i * 4 + l) * 6];
        for (int a = 0; a < 6; ++a) {
          if (u[a] == 0.0) continue;
          for (int b = 0; b < 6; ++b)
            if (w[b] != 0.0) s += u[a] * w[b] * Z[6 * a + b];
        }
      }
      tot[4 * j + l] = s;
    }
  double ev[4], vec[16];
  mb2::jacobi_eigen<4>(tot, ev, vec);
  q[0] = vec[4 * 1 + 0];
  q[1] = vec[4 * 2 + 0];
  q[2] = vec[4 * 3 + 0];
  q[3] = vec[4 * 0 + 0];
}

int main() {
  std::mt19937_64 g(11);
  std::uniform_real_distribution<double> U(-1e3, 1e3);
  long bad = 0;
  const int n = 20000;
  for (int t = 0; t < n; ++t) {
    double Z[36];
    const double scale = t % 7 == 0 ? 1e-9 : (t % 5 == 0 ? 1e6 : 1.0);
    for (double &z : Z) z = U(g) * scale;
    if (t % 11 == 0) Z[t % 36] = 0.0;
    if (t % 13 == 0) Z[(t + 5) % 36] = -0.0;
    double q0[4], q1[4];
    horn_table(Z, q0);
    mb2::horn_quaternion(Z, q1);
    if (std::memcmp(q0, q1, sizeof(q0)) != 0) ++bad;
  }
  std::printf("%ld\n", bad);
  return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_horn_terms_equal_coefficient_table(tmp_path):
    src = tmp_path / "horn.cpp"
    src.write_text(SRC)
    exe = tmp_path / "horn"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-x", "c++",
                           "-I", os.path.join(ROOT, "mirorr_b200", "csrc"),
                           "-I", os.path.join(ROOT, "include"),
                           "-D__host__=", "-D__device__=", "-D__forceinline__=inline",
                           str(src), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert int(out.strip()) == 0


SRC_SQRT = r'''
#include <cstdio>
#include <cmath>
#include <random>
#include <initializer_list>
#include "tfm.cuh"

// Denman-Beavers half transform: sqrt(M)^2 = M for homogeneous affine M near
// the identity, and the affine inverse undoes M.
int main() {
  std::mt19937_64 g(5);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  double worst_sq = 0.0, worst_inv = 0.0;
  for (int t = 0; t < 2000; ++t) {
    double m[16] = {0};
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) m[4 * r + c] = (r == c ? 1.0 : 0.0) + 0.08 * U(g);
      m[4 * r + 3] = 12.0 * U(g);
    }
    m[15] = 1.0;
    double h[16], hh[16], mi[16], id[16];
    mb2::matrix_sqrt4(m, h);
    mb2::mn_mul<4>(h, h, hh);
    for (int i = 0; i < 16; ++i) worst_sq = std::fmax(worst_sq, std::fabs(hh[i] - m[i]));
    if (!mb2::affine4_inverse(m, mi)) return 2;
    mb2::mn_mul<4>(m, mi, id);
    for (int i = 0; i < 16; ++i)
      worst_inv = std::fmax(worst_inv, std::fabs(id[i] - (i % 5 == 0 ? 1.0 : 0.0)));
  }
  std::printf("%.3e %.3e\n", worst_sq, worst_inv);
  return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_half_transform_and_affine_inverse(tmp_path):
    """matrix_sqrt4 (Denman-Beavers, vnl_utils.h:46-95) squares back to its
    input and affine4_inverse inverts, to FP64 rounding, on 2,000 random
    homogeneous affine matrices near the identity (rotation/scale entries
    within 0.08 of it, translations up to 12 mm)."""
    src = tmp_path / "sqrt.cpp"
    src.write_text(SRC_SQRT)
    exe = tmp_path / "sqrt"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-x", "c++",
                           "-I", os.path.join(ROOT, "mirorr_b200", "csrc"),
                           "-I", os.path.join(ROOT, "include"),
                           "-D__host__=", "-D__device__=", "-D__forceinline__=inline",
                           str(src), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sq, inv = (float(v) for v in r.stdout.split())
    assert sq < 1e-12 and inv < 1e-12, (sq, inv)
