// nifti_io.cpp -- NIfTI-1 reader / writer (see nifti_io.hpp).
#include "nifti_io.hpp"

#include <zlib.h>

#include <cmath>
#include <cstring>
#include <stdexcept>

namespace mirorr_cli {

namespace {

constexpr int kHdr = 348;

template <class T>
T get(const unsigned char *h, int off, bool swap) {
  T v;
  unsigned char b[sizeof(T)];
  std::memcpy(b, h + off, sizeof(T));
  if (swap)
    for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(b[i], b[sizeof(T) - 1 - i]);
  std::memcpy(&v, b, sizeof(T));
  return v;
}

template <class T>
void put(unsigned char *h, int off, T v) {
  std::memcpy(h + off, &v, sizeof(T));
}

struct GzFile {
  gzFile f = nullptr;
  GzFile(const std::string &path, const char *mode) : f(gzopen(path.c_str(), mode)) {}
  ~GzFile() {
    if (f) gzclose(f);
  }
};

bool ends_with(const std::string &s, const std::string &t) {
  return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

// geometry of a voxel-to-RAS affine (3x3 part A, translation t), converted to LPS
void geom_from_ras(const double A[3][3], const double t[3], mirorr_geometry &g) {
  for (int c = 0; c < 3; ++c) {
    double n = std::sqrt(A[0][c] * A[0][c] + A[1][c] * A[1][c] + A[2][c] * A[2][c]);
    if (!(n > 0.0)) n = 1.0;
    g.spacing[c] = n;
    for (int r = 0; r < 3; ++r) g.direction[3 * r + c] = A[r][c] / n;
  }
  for (int r = 0; r < 3; ++r) g.origin[r] = t[r];
  for (int r = 0; r < 2; ++r) {
    g.origin[r] = -g.origin[r];
    for (int c = 0; c < 3; ++c) g.direction[3 * r + c] = -g.direction[3 * r + c];
  }
}

void write_nifti(const std::string &path, const mirorr_geometry &g, const void *data,
                 short datatype, short bitpix) {
  unsigned char h[kHdr + 4];
  std::memset(h, 0, sizeof(h));
  put<int>(h, 0, kHdr);
  short dim[8] = {3, (short)g.size[0], (short)g.size[1], (short)g.size[2], 1, 1, 1, 1};
  for (int i = 0; i < 8; ++i) put<short>(h, 40 + 2 * i, dim[i]);
  put<short>(h, 70, datatype);
  put<short>(h, 72, bitpix);
  // RAS direction and origin
  double D[3][3], o[3];
  for (int r = 0; r < 3; ++r) {
    const double sgn = r < 2 ? -1.0 : 1.0;
    for (int c = 0; c < 3; ++c) D[r][c] = sgn * g.direction[3 * r + c];
    o[r] = sgn * g.origin[r];
  }
  const double det = D[0][0] * (D[1][1] * D[2][2] - D[1][2] * D[2][1]) -
                     D[0][1] * (D[1][0] * D[2][2] - D[1][2] * D[2][0]) +
                     D[0][2] * (D[1][0] * D[2][1] - D[1][1] * D[2][0]);
  const double qfac = det < 0.0 ? -1.0 : 1.0;
  float pixdim[8] = {(float)qfac, (float)g.spacing[0], (float)g.spacing[1], (float)g.spacing[2],
                     0, 0, 0, 0};
  for (int i = 0; i < 8; ++i) put<float>(h, 76 + 4 * i, pixdim[i]);
  put<float>(h, 108, (float)(kHdr + 4));
  put<float>(h, 112, 1.0f);
  h[123] = 2;  // mm
  put<short>(h, 252, 1);
  put<short>(h, 254, 1);
  // quaternion of the rotation (third column scaled by qfac); Shepperd's method
  double R[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) R[r][c] = D[r][c] * (c == 2 ? qfac : 1.0);
  double a, b, c, d;
  const double tr = R[0][0] + R[1][1] + R[2][2];
  if (tr > 0.0) {
    const double s = 0.5 / std::sqrt(tr + 1.0);
    a = 0.25 / s; b = (R[2][1] - R[1][2]) * s; c = (R[0][2] - R[2][0]) * s; d = (R[1][0] - R[0][1]) * s;
  } else if (R[0][0] > R[1][1] && R[0][0] > R[2][2]) {
    const double s = 2.0 * std::sqrt(1.0 + R[0][0] - R[1][1] - R[2][2]);
    a = (R[2][1] - R[1][2]) / s; b = 0.25 * s; c = (R[0][1] + R[1][0]) / s; d = (R[0][2] + R[2][0]) / s;
  } else if (R[1][1] > R[2][2]) {
    const double s = 2.0 * std::sqrt(1.0 + R[1][1] - R[0][0] - R[2][2]);
    a = (R[0][2] - R[2][0]) / s; b = (R[0][1] + R[1][0]) / s; c = 0.25 * s; d = (R[1][2] + R[2][1]) / s;
  } else {
    const double s = 2.0 * std::sqrt(1.0 + R[2][2] - R[0][0] - R[1][1]);
    a = (R[1][0] - R[0][1]) / s; b = (R[0][2] + R[2][0]) / s; c = (R[1][2] + R[2][1]) / s; d = 0.25 * s;
  }
  if (a < 0.0) { b = -b; c = -c; d = -d; }
  put<float>(h, 256, (float)b);
  put<float>(h, 260, (float)c);
  put<float>(h, 264, (float)d);
  for (int r = 0; r < 3; ++r) put<float>(h, 268 + 4 * r, (float)o[r]);
  for (int r = 0; r < 3; ++r) {
    for (int cc = 0; cc < 3; ++cc) put<float>(h, 280 + 16 * r + 4 * cc, (float)(D[r][cc] * g.spacing[cc]));
    put<float>(h, 280 + 16 * r + 12, (float)o[r]);
  }
  std::memcpy(h + 344, "n+1\0", 4);
  GzFile f(path, ends_with(path, ".gz") ? "wb6" : "wbT");
  if (!f.f) throw std::runtime_error("cannot write " + path);
  const size_t bytes = (size_t)g.size[0] * g.size[1] * g.size[2] * (bitpix / 8);
  if (gzwrite(f.f, h, sizeof(h)) != (int)sizeof(h) ||
      gzwrite(f.f, data, (unsigned)bytes) != (int)bytes)
    throw std::runtime_error("write failed: " + path);
}

}  // namespace

Volume read_nifti(const std::string &path) {
  GzFile f(path, "rb");
  if (!f.f) throw std::runtime_error("cannot open " + path);
  unsigned char h[kHdr];
  if (gzread(f.f, h, kHdr) != kHdr) throw std::runtime_error("short NIfTI header: " + path);
  bool swap = false;
  if (get<int>(h, 0, false) != kHdr) {
    swap = true;
    if (get<int>(h, 0, true) != kHdr) throw std::runtime_error("not a NIfTI-1 file: " + path);
  }
  short dim[8];
  for (int i = 0; i < 8; ++i) dim[i] = get<short>(h, 40 + 2 * i, swap);
  if (dim[0] < 3 || dim[1] < 1 || dim[2] < 1 || dim[3] < 1)
    throw std::runtime_error("not a 3D volume: " + path);
  const short datatype = get<short>(h, 70, swap);
  float pixdim[8];
  for (int i = 0; i < 8; ++i) pixdim[i] = get<float>(h, 76 + 4 * i, swap);
  const float vox_offset = get<float>(h, 108, swap);
  float slope = get<float>(h, 112, swap), inter = get<float>(h, 116, swap);
  if (slope == 0.0f || !std::isfinite(slope)) { slope = 1.0f; inter = 0.0f; }
  const short qcode = get<short>(h, 252, swap), scode = get<short>(h, 254, swap);

  Volume v;
  mirorr_geometry &g = v.geom;
  g.size[0] = dim[1]; g.size[1] = dim[2]; g.size[2] = dim[3];
  double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, t[3] = {0, 0, 0};
  const double dx = std::fabs(pixdim[1]) > 0 ? std::fabs(pixdim[1]) : 1.0;
  const double dy = std::fabs(pixdim[2]) > 0 ? std::fabs(pixdim[2]) : 1.0;
  const double dz = std::fabs(pixdim[3]) > 0 ? std::fabs(pixdim[3]) : 1.0;
  if (qcode > 0) {
    const double b = get<float>(h, 256, swap), c = get<float>(h, 260, swap),
                 d = get<float>(h, 264, swap);
    double a = 1.0 - (b * b + c * c + d * d);
    a = a > 0.0 ? std::sqrt(a) : 0.0;
    const double qfac = pixdim[0] < 0.0f ? -1.0 : 1.0;
    const double R[3][3] = {{a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)},
                            {2 * (b * c + a * d), a * a + c * c - b * b - d * d, 2 * (c * d - a * b)},
                            {2 * (b * d - a * c), 2 * (c * d + a * b), a * a + d * d - b * b - c * c}};
    for (int r = 0; r < 3; ++r) {
      A[r][0] = R[r][0] * dx;
      A[r][1] = R[r][1] * dy;
      A[r][2] = R[r][2] * dz * qfac;
      t[r] = get<float>(h, 268 + 4 * r, swap);
    }
  } else if (scode > 0) {
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) A[r][c] = get<float>(h, 280 + 16 * r + 4 * c, swap);
      t[r] = get<float>(h, 280 + 16 * r + 12, swap);
    }
  } else {
    A[0][0] = dx; A[1][1] = dy; A[2][2] = dz;
  }
  geom_from_ras(A, t, g);

  const size_t n = (size_t)g.size[0] * g.size[1] * g.size[2];
  int bytes = 0;
  switch (datatype) {
    case 2: case 256: bytes = 1; break;
    case 4: case 512: bytes = 2; break;
    case 8: case 16: case 768: bytes = 4; break;
    case 64: bytes = 8; break;
    default: throw std::runtime_error("unsupported NIfTI datatype " + std::to_string(datatype) + ": " + path);
  }
  const long off = vox_offset >= (float)kHdr ? (long)vox_offset : kHdr + 4;
  if (gzseek(f.f, off, SEEK_SET) != off) throw std::runtime_error("bad vox_offset: " + path);
  std::vector<unsigned char> raw(n * bytes);
  const size_t chunk = 1u << 30;
  for (size_t done = 0; done < raw.size();) {
    const unsigned want = (unsigned)std::min(chunk, raw.size() - done);
    if (gzread(f.f, raw.data() + done, want) != (int)want)
      throw std::runtime_error("short voxel data: " + path);
    done += want;
  }
  if (swap && bytes > 1)
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < bytes / 2; ++j) std::swap(raw[i * bytes + j], raw[i * bytes + bytes - 1 - j]);
  v.data.resize(n);
  const unsigned char *p = raw.data();
  for (size_t i = 0; i < n; ++i) {
    double x = 0.0;
    switch (datatype) {
      case 2: x = p[i]; break;
      case 256: x = (int8_t)p[i]; break;
      case 4: { int16_t q; std::memcpy(&q, p + 2 * i, 2); x = q; } break;
      case 512: { uint16_t q; std::memcpy(&q, p + 2 * i, 2); x = q; } break;
      case 8: { int32_t q; std::memcpy(&q, p + 4 * i, 4); x = q; } break;
      case 768: { uint32_t q; std::memcpy(&q, p + 4 * i, 4); x = q; } break;
      case 16: { float q; std::memcpy(&q, p + 4 * i, 4); x = q; } break;
      case 64: { double q; std::memcpy(&q, p + 8 * i, 8); x = q; } break;
    }
    v.data[i] = (float)(x * slope + inter);
  }
  return v;
}

void write_nifti_float(const std::string &path, const mirorr_geometry &g, const float *data) {
  write_nifti(path, g, data, 16, 32);
}

void write_nifti_u8(const std::string &path, const mirorr_geometry &g, const uint8_t *data) {
  write_nifti(path, g, data, 2, 8);
}

}  // namespace mirorr_cli
