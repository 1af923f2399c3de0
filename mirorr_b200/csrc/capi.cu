// capi.cu -- C ABI of mirorr_b200 (declared in include/mirorr_b200.h):
// context, block matcher (the AbstractBlockMatcher replacement), resampler,
// LTS fit, pyramid, and the device-resident registration driver
// (MirorrPyramidImplement::RunMirorr + the classic / symmetric iteration loops).
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <iterator>
#include <map>
#include <mutex>
#include <vector>

#include <cuda.h>

#include "kernels.cuh"

namespace mb2 {

static thread_local char t_err[512] = "";
int64_t g_launches = 0;

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
}
void clear_error() { t_err[0] = 0; }
const char *get_error() { return t_err; }

int sm_count() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 148;
  }
  if (dev >= 0 && dev < 64) {
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
  }
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = 148;
  }
  if (dev >= 0 && dev < 64) cached[dev].store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace mb2

using namespace mb2;

// Per-stage timing of matcher calls, accumulated from CUDA events.
struct StageTimer {
  static constexpr size_t kPerCall = 7;  // 5 stage boundaries + the search kernel's 2
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  double ms[4] = {0, 0, 0, 0};
  long long calls = 0;
  double search_ms = 0.0;     // the FP32 search kernel (events 5, 6 of a call)
  long long search_calls = 0;
  std::vector<char> ran;      // per call: the search kernel ran (events 5, 6 recorded)
  // resampler passes (an image and its mask into one middle-space grid)
  std::vector<cudaEvent_t> rpool;
  size_t rused = 0;
  std::vector<long long> rvox;
  double resample_ms = 0.0;
  long long resample_passes = 0, resample_voxels = 0;
  cudaEvent_t *take_resample(long long voxels) {
    while (rpool.size() < rused + 2) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      rpool.push_back(e);
    }
    cudaEvent_t *p = &rpool[rused];
    rused += 2;
    rvox.push_back(voxels);
    return p;
  }
  cudaEvent_t *take(size_t k) {
    while (pool.size() < used + k) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      pool.push_back(e);
    }
    cudaEvent_t *p = &pool[used];
    used += k;
    return p;
  }
  // call after a stream synchronize
  void harvest() {
    for (size_t i = 0; i + kPerCall <= used; i += kPerCall) {
      for (int s = 0; s < 4; ++s) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, pool[i + s], pool[i + s + 1]) == cudaSuccess) ms[s] += t;
      }
      const size_t j = i / kPerCall;
      float t = 0.f;
      if (j < ran.size() && ran[j] &&
          cudaEventElapsedTime(&t, pool[i + 5], pool[i + 6]) == cudaSuccess) {
        search_ms += t;
        ++search_calls;
      }
      ++calls;
    }
    ran.clear();
    used = 0;
    for (size_t i = 0; i + 2 <= rused; i += 2) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, rpool[i], rpool[i + 1]) == cudaSuccess) {
        resample_ms += t;
        ++resample_passes;
        resample_voxels += rvox[i / 2];
      }
    }
    rused = 0;
    rvox.clear();
    cudaGetLastError();
  }
  void release() {
    for (auto e : pool) cudaEventDestroy(e);
    for (auto e : rpool) cudaEventDestroy(e);
    rpool.clear();
    rvox.clear();
    rused = 0;
    pool.clear();
    ran.clear();
    used = 0;
  }
};

struct mirorr_ctx_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches0 = 0;
  BmWork bmw;
  Bm16Work bm16;
  LtsWork ltsw;
  DevBuf counts;      // long long[4]
  DevBuf ncc_count;   // unsigned long long
  DevBuf ones;        // default all-255 mask
  long long ones_n = 0;
  StageTimer timer;
  DevBuf xl_count;    // unsigned long long: candidates scored by the search kernel
  // registration scratch
  DevBuf lvl_f, lvl_m, tmp_a, tmp_b, weights;
  DevBuf img_b, img_s, msk_b, msk_s;
  DevBuf best, second, match, status;
  DevBuf pts_i, pts_m;
  DevBuf up_f, up_m, up_fm, up_mm;
  // iteration graphs of the float32 registration: the resampling jobs and the
  // fit's state travel through pinned staging; one executable graph per
  // pyramid level, kept for the next registration while its key (geometry,
  // parameters, every buffer its launches address) is unchanged
  HostBuf it_jobs, it_lts_in, it_lts_out;
  DevBuf it_jobs_d;
  bool graphs = true;
  struct LevelGraph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
  };
  LevelGraph lgraph[16];
};

struct Vol {
  const void *img = nullptr;     // element type: the matcher's storage

  const uint8_t *mask = nullptr;
  DevBuf own_img, own_mask;
  bool has = false;
  bool has_mask = false;
  mirorr_geometry geom{};
};

struct mirorr_matcher_s {
  mirorr_ctx ctx = nullptr;
  mirorr_bm_params p{};
  int storage = MIRORR_DTYPE_F32;  // element type of the stored images
  Vol base, search;
  DevBuf best, second, match, status, pts_b, pts_m;
  BmGeom last{};
  bool has_results = false;
  long long kept = 0;
  cudaEvent_t ev[5] = {};
  float timings[4] = {0, 0, 0, 0};
};

namespace {

size_t elem_size(int dtype) { return dtype == MIRORR_DTYPE_F32 ? 4 : (dtype == MIRORR_DTYPE_U8 ? 1 : 2); }
bool is16(int dtype) { return dtype == MIRORR_DTYPE_BF16 || dtype == MIRORR_DTYPE_F16; }

mirorr_status check_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device available (%s)",
              e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    return MIRORR_ECUDA;
  }
  if (device < 0 || device >= n) {
    set_error("device %d out of range (%d devices)", device, n);
    return MIRORR_EINVAL;
  }
  cudaDeviceProp prop;
  MB2_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a (B200)", device,
              prop.major, prop.minor);
    return MIRORR_ECUDA;
  }
  return MIRORR_OK;
}

bool valid_geom(const mirorr_geometry *g) {
  if (!g) return false;
  for (int d = 0; d < 3; ++d)
    if (g->size[d] <= 0 || !(g->spacing[d] > 0.0)) return false;
  // the resampler addresses within a slice with 32-bit offsets
  if ((long long)g->size[0] * g->size[1] >= (1LL << 31)) return false;
  double A[9], Ai[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[3 * r + c] = g->direction[3 * r + c] * g->spacing[c];
  return mn_inverse<3>(A, Ai);
}

mirorr_status ensure_ones(mirorr_ctx c, long long n) {
  if (c->ones_n >= n) return MIRORR_OK;
  MB2_TRY(c->ones.ensure(n));
  MB2_TRY(launch_fill_u8(c->ones.as<uint8_t>(), n, 255, c->stream));
  c->ones_n = n;
  return MIRORR_OK;
}

void index_to_physical(const mirorr_geometry &g, double *A) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[3 * r + c] = g.direction[3 * r + c] * g.spacing[c];
}

// out index -> in continuous index: C = Ain^-1 M Aout, e = Ain^-1 (M Oout + off - Oin)
bool make_map(const mirorr_geometry &out, const mirorr_geometry &in, const double *M,
              const double *off, ResampleMap &m) {
  double Aout[9], Ain[9], Ainv[9], MA[9], v[3], w[3];
  index_to_physical(out, Aout);
  index_to_physical(in, Ain);
  if (!mn_inverse<3>(Ain, Ainv)) return false;
  m3_mul(M, Aout, MA);
  m3_mul(Ainv, MA, m.C);
  m3_vec(M, out.origin, v);
  for (int i = 0; i < 3; ++i) w[i] = v[i] + off[i] - in.origin[i];
  m3_vec(Ainv, w, m.e);
  return true;
}

void center_of(const mirorr_geometry &g, double *c) {
  double A[9], ci[3];
  index_to_physical(g, A);
  for (int d = 0; d < 3; ++d) ci[d] = ((double)g.size[d] - 1.0) / 2.0;
  m3_vec(A, ci, c);
  for (int d = 0; d < 3; ++d) c[d] += g.origin[d];
}

void to_public(const Tfm &t, mirorr_transform &o) {
  o.kind = t.kind;
  for (int i = 0; i < 9; ++i) o.matrix[i] = t.M[i];
  for (int i = 0; i < 3; ++i) { o.offset[i] = t.off[i]; o.center[i] = t.c[i]; }
  for (int i = 0; i < 12; ++i) o.params[i] = 0.0;
  tfm_params(t, o.params);
}

bool from_public(const mirorr_transform &o, Tfm &t) {
  if (o.kind != KIND_RIGID && o.kind != KIND_AFFINE) return false;
  tfm_identity(t, o.kind);
  tfm_set_center(t, o.center);
  tfm_set_params(t, o.params);
  return true;
}

mirorr_status check_bm_params(const mirorr_bm_params &p) {
  if (p.block_width < 1 || p.block_width > 8) {
    set_error("block_width %u not supported (1..8)", p.block_width);
    return MIRORR_EINVAL;
  }
  if (p.block_gap < 1 || p.nhood_gap < 1 || p.nhood_width < 1) {
    set_error("block_gap, nhood_gap and nhood_width must be >= 1");
    return MIRORR_EINVAL;
  }
  double pk = p.portion_matches_kept;
  if (pk < 0.0 || pk > 1.0 || pk != pk) {
    set_error("PortionMatchesKept is %g. It should be between 0 and 1.0.", pk);
    return MIRORR_EINVAL;
  }
  if (!(p.block_keep > 0.0)) {
    set_error("block_keep must be > 0 (>= 1 keeps every block)");
    return MIRORR_EINVAL;
  }
  int e = ((int)p.nhood_width - 1) * (int)p.block_gap + (int)p.block_width;
  size_t smem = (size_t)e * e * e * 5 + 1024;
  if (e > 40 || smem > 200 * 1024) {
    set_error("search window too large: (nhood_width-1)*block_gap+block_width = %d", e);
    return MIRORR_EINVAL;
  }
  return MIRORR_OK;
}

// ---- one matcher call on device data ---------------------------------------
struct MatchCall {
  const void *base, *search;   // element type `dtype`
  int dtype;
  const uint8_t *bmask, *smask;
  int size[3];
  mirorr_geometry point_geom;  // base image geometry (blockPositionToPoint)
};

mirorr_status run_match(mirorr_ctx c, const mirorr_bm_params &p, const MatchCall &mc,
                        BmGeom &g, DevBuf &best, DevBuf &second, DevBuf &match,
                        DevBuf &status, double *pts_b, double *pts_m, long long *count_dev,
                        const long long *offset_dev, cudaEvent_t *ev,
                        cudaEvent_t *kev = nullptr, unsigned long long *xl_count = nullptr,
                        bool *xl_ran = nullptr) {
  if (!bm_geometry(mc.size, (int)p.block_width, (int)p.block_gap, (int)p.nhood_gap,
                   (int)p.nhood_width, g)) {
    set_error("image smaller than one block or invalid block parameters");
    return MIRORR_EINVAL;
  }
  long long nvox = (long long)mc.size[0] * mc.size[1] * mc.size[2];
  if (!is16(mc.dtype)) MB2_TRY(c->bmw.stats.ensure(sizeof(float2) * nvox));
  MB2_TRY(best.ensure(sizeof(float) * g.nblocks));
  MB2_TRY(second.ensure(sizeof(float) * g.nblocks));
  MB2_TRY(match.ensure(sizeof(int32_t) * g.nblocks));
  MB2_TRY(status.ensure(g.nblocks));
  cudaStream_t s = c->stream;
  BmOut out{best.as<float>(), second.as<float>(), match.as<int32_t>(), status.as<uint8_t>()};
  if (is16(mc.dtype)) {
    // 16-bit storage: box statistics, selection and search of tc.cu
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[0], s));
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[1], s));
    const uint8_t *sel = nullptr;
    unsigned int *give_up = nullptr;
    if (p.block_keep < 1.0) MB2_TRY(ncc_give_up_flag(c->bmw, s, &give_up));
    MB2_TRY(launch_variance_selection(g, mc.base, p.block_keep, c->bmw, &sel, s, mc.dtype,
                                      give_up, c->ltsw.spin_limit));
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[2], s));
    MB2_TRY(launch_match16(mc.dtype, g, mc.base, mc.bmask, mc.search, mc.smask, sel, out, c->bm16,
                           c->ncc_count.as<unsigned long long>(), s));
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[3], s));
    if (xl_ran) *xl_ran = false;
  } else {
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[0], s));
    MB2_TRY(launch_box_stats(g, static_cast<const float *>(mc.search), mc.smask,
                             c->bmw.stats.as<float2>(), s));
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[1], s));
    const uint8_t *sel = nullptr;
    unsigned int *give_up = nullptr;
    if (p.block_keep < 1.0) MB2_TRY(ncc_give_up_flag(c->bmw, s, &give_up));
    MB2_TRY(launch_variance_selection(g, mc.base, p.block_keep, c->bmw, &sel, s,
                                      MIRORR_DTYPE_F32, give_up, c->ltsw.spin_limit));
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[2], s));
    MB2_TRY(launch_ncc(g, static_cast<const float *>(mc.base), mc.bmask,
                       static_cast<const float *>(mc.search), mc.smask, c->bmw.stats.as<float2>(),
                       sel, out, c->bmw, c->ncc_count.as<unsigned long long>(), s, kev, xl_count,
                       xl_ran));
    if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[3], s));
  }
  PointGeom pg;
  point_geom(mc.point_geom.origin, mc.point_geom.spacing, mc.point_geom.direction,
             (int)p.block_width, pg);
  MB2_TRY(launch_postfilter(g, out, c->bmw, pg, pts_b, pts_m, count_dev, offset_dev, s));
  if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[4], s));
  return MIRORR_OK;
}

// ---- pyramid schedule: PyramidScheduleTuner::UpdateSymmetric -----------------
double num_octaves(double dim, double base) { return std::floor(std::log(dim / base) / std::log(2.0)); }
unsigned num_levels(double dim, double base) {
  return 1u + (unsigned)std::max(0.0, num_octaves(dim, base));
}
unsigned best_rate(double big, double small) {
  unsigned e = (unsigned)std::max(0.0, num_octaves(big * (4.0 / 3.0), small));
  return 1u << e;
}

int pyramid_schedule(const mirorr_geometry &fg, const mirorr_geometry &mg, int min_length,
                     int max_levels, int sm_out[16][3], int sf_out[16][3]) {
  double ml = std::max({mg.size[0], mg.size[1], mg.size[2]});
  double fl = std::max({fg.size[0], fg.size[1], fg.size[2]});
  int mpl = 1 + (int)std::max(num_levels(ml, min_length), num_levels(fl, min_length));
  std::vector<std::array<long long, 3>> sm(mpl), sf(mpl);
  for (auto &r : sm) r = {-1, -1, -1};
  for (auto &r : sf) r = {-1, -1, -1};
  for (int d = 0; d < 3; ++d) {
    int r = 1;
    sm[mpl - r][d] = 1;
    sf[mpl - r][d] = 1;
    double mb = mg.spacing[d], fb = fg.spacing[d];
    long long me = 1LL << (num_levels(mg.size[d], min_length) - 1);
    long long fe = 1LL << (num_levels(fg.size[d], min_length) - 1);
    r = 2;
    if (mb < fb) {
      long long rate = std::min<long long>(best_rate(fb, mb), me);
      for (long long s = rate >= 2 ? 2 : 1; s <= rate; s *= 2) {
        sm[mpl - r][d] = s; sf[mpl - r][d] = 1; ++r;
      }
    } else if (mb > fb) {
      long long rate = std::min<long long>(best_rate(mb, fb), fe);
      for (long long s = rate >= 2 ? 2 : 1; s <= rate; s *= 2) {
        sm[mpl - r][d] = 1; sf[mpl - r][d] = s; ++r;
      }
    } else {
      sm[mpl - r][d] = 1; sf[mpl - r][d] = 1; ++r;
    }
    for (int lev = mpl - r; lev >= 0; --lev) {
      if (2 * sm[lev + 1][d] > me || 2 * sf[lev + 1][d] > fe) {
        sm[lev][d] = sm[lev + 1][d]; sf[lev][d] = sf[lev + 1][d];
      } else {
        sm[lev][d] = 2 * sm[lev + 1][d]; sf[lev][d] = 2 * sf[lev + 1][d];
      }
    }
  }
  int first = 0;
  {
    int nd = 0;
    for (int d = 0; d < 3; ++d) {
      if (sm[mpl - 1][d] != sm[mpl - 2][d]) ++nd;
      if (sf[mpl - 1][d] != sf[mpl - 2][d]) ++nd;
    }
    if (nd == 0) first = 1;
  }
  int last = mpl;
  for (int lev = 2; lev < mpl; ++lev) {
    int nd = 0;
    for (int d = 0; d < 3; ++d) {
      if (sm[mpl - lev - 1][d] != sm[mpl - lev][d]) ++nd;
      if (sf[mpl - lev - 1][d] != sf[mpl - lev][d]) ++nd;
    }
    if (nd < 3) { last = lev; break; }
  }
  int n = last - first;
  if (max_levels > 0 && n > max_levels) n = max_levels;
  if (n > 16) n = 16;
  for (int lev = 0; lev < n; ++lev)
    for (int d = 0; d < 3; ++d) {
      sm_out[n - lev - 1][d] = (int)sm[mpl - first - lev - 1][d];
      sf_out[n - lev - 1][d] = (int)sf[mpl - first - lev - 1][d];
    }
  return n;
}

// Gaussian of sigma = f/2 voxels, radius ceil(3 sigma), normalised by the
// sequential sum.
int gaussian_weights(int f, double *w) {
  if (f <= 1) { w[0] = 1.0; return 0; }
  double sigma = f / 2.0;
  int r = (int)std::ceil(3.0 * sigma);
  double s = 0.0;
  for (int k = -r; k <= r; ++k) {
    w[k + r] = std::exp(-((double)k * (double)k) / (2.0 * sigma * sigma));
  }
  for (int k = 0; k <= 2 * r; ++k) s += w[k];
  for (int k = 0; k <= 2 * r; ++k) w[k] = w[k] / s;
  return r;
}

void level_geometry(const mirorr_geometry &in, const int f[3], mirorr_geometry &out) {
  out = in;
  double ds[3];
  for (int d = 0; d < 3; ++d) {
    out.size[d] = std::max(1, (int)std::floor((double)in.size[d] / (double)f[d]));
    out.spacing[d] = in.spacing[d] * (double)f[d];
    ds[d] = (out.spacing[d] - in.spacing[d]) * 0.5;
  }
  double v[3];
  m3_vec(in.direction, ds, v);
  for (int d = 0; d < 3; ++d) out.origin[d] = in.origin[d] + v[d];
}

// Builds one pyramid level on the device.  When every factor is 1 the input
// itself is the level (*out_ptr = in, no copy, the input's element type);
// otherwise the level is float32 (the first smoothing pass reads the input's
// type).
mirorr_status make_level(mirorr_ctx c, const mirorr_geometry &ig, const void *in, int in_dtype,
                         const int f[3], mirorr_geometry &og, DevBuf &out, const void **out_ptr,
                         int *out_dtype) {
  level_geometry(ig, f, og);
  if (f[0] == 1 && f[1] == 1 && f[2] == 1) {
    *out_ptr = in;
    *out_dtype = in_dtype;
    return MIRORR_OK;
  }
  cudaStream_t s = c->stream;
  long long n = vox(ig.size);
  MB2_TRY(c->tmp_a.ensure(sizeof(float) * n));
  MB2_TRY(c->tmp_b.ensure(sizeof(float) * n));
  MB2_TRY(c->weights.ensure(sizeof(double) * 3 * 64));
  double w[3][64];
  int rad[3];
  for (int d = 0; d < 3; ++d) {
    if (f[d] > 20) {
      set_error("pyramid factor %d too large", f[d]);
      return MIRORR_EINVAL;
    }
    rad[d] = gaussian_weights(f[d], w[d]);
  }
  MB2_CUDA_TRY(cudaMemcpyAsync(c->weights.ptr, w, sizeof(w), cudaMemcpyHostToDevice, s));
  const void *cur = in;
  int cur_t = in_dtype;
  float *bufs[2] = {c->tmp_a.as<float>(), c->tmp_b.as<float>()};
  int bi = 0;
  for (int d = 0; d < 3; ++d) {
    if (f[d] <= 1) continue;
    MB2_TRY(launch_smooth_axis(ig.size, cur, bufs[bi], d, c->weights.as<double>() + 64 * d,
                               rad[d], s, cur_t));
    cur = bufs[bi];
    cur_t = MIRORR_DTYPE_F32;
    bi ^= 1;
  }
  MB2_TRY(out.ensure(sizeof(float) * vox(og.size)));
  ResampleMap m;
  for (int i = 0; i < 9; ++i) m.C[i] = 0.0;
  for (int d = 0; d < 3; ++d) {
    m.C[4 * d] = (double)f[d];
    m.e[d] = ((double)f[d] - 1.0) / 2.0;
  }
  if (cur_t != MIRORR_DTYPE_F32) {
    set_error("a pyramid factor above 1 on some axis is required to smooth a 16-bit level");
    return MIRORR_EINVAL;
  }
  MB2_TRY(launch_resample(ig.size, cur, nullptr, og.size, m, out.as<float>(), nullptr, s));
  *out_ptr = out.as<float>();
  *out_dtype = MIRORR_DTYPE_F32;
  return MIRORR_OK;
}

// ---- registration ----------------------------------------------------------
struct RegImage {
  const void *img;
  int dtype;        // element type of img
  mirorr_geometry g;
};

struct RegRun {
  mirorr_ctx c;
  const mirorr_reg_params *p;
  const uint8_t *fmask;   // full resolution
  const uint8_t *mmask;
  mirorr_geometry fmask_g, mmask_g;
  mirorr_reg_stats *stats;
  int level;
};

mirorr_status resample_into(mirorr_ctx c, const RegImage &src, const uint8_t *mask,
                            const mirorr_geometry &mask_g, const mirorr_geometry &grid,
                            const Tfm &t, DevBuf &img, DevBuf &msk, int out_dtype) {
  ResampleMap mi, mm;
  if (!make_map(grid, src.g, t.M, t.off, mi) || !make_map(grid, mask_g, t.M, t.off, mm)) {
    set_error("singular image geometry");
    return MIRORR_EINVAL;
  }
  long long n = vox(grid.size);
  MB2_TRY(img.ensure(elem_size(out_dtype) * n));
  MB2_TRY(msk.ensure(n));
  cudaEvent_t *ev = c->timer.on ? c->timer.take_resample(n) : nullptr;
  if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[0], c->stream));
  const bool same_grid = src.g.size[0] == mask_g.size[0] && src.g.size[1] == mask_g.size[1] &&
                         src.g.size[2] == mask_g.size[2] && memcmp(&mi, &mm, sizeof(mi)) == 0;
  // the default mask (no mask given) is 255 everywhere and is not read
  const bool ones = c->ones.ptr && mask == c->ones.as<uint8_t>();
  if (same_grid) {
    // image and mask on one input grid (the finest level): one pass computes
    // each voxel's index map once for both
    MB2_TRY(launch_resample(src.g.size, src.img, mask, grid.size, mi, img.ptr, msk.as<uint8_t>(),
                            c->stream, false, src.dtype, out_dtype, ones));
  } else {
    MB2_TRY(launch_resample(src.g.size, src.img, nullptr, grid.size, mi, img.ptr, nullptr,
                            c->stream, false, src.dtype, out_dtype));
    MB2_TRY(launch_resample(mask_g.size, nullptr, mask, grid.size, mm, nullptr,
                            msk.as<uint8_t>(), c->stream, false, MIRORR_DTYPE_F32, MIRORR_DTYPE_F32,
                            ones));
  }
  if (ev) MB2_CUDA_TRY(cudaEventRecord(ev[1], c->stream));
  return MIRORR_OK;
}

// The resampling jobs resample_into launches for (src, mask) onto grid through
// t, appended to jobs[nj..]: one image + mask job on a shared input grid,
// else an image job and a mask job (float32 images only).
mirorr_status make_jobs(mirorr_ctx c, const RegImage &src, const uint8_t *mask,
                        const mirorr_geometry &mask_g, const mirorr_geometry &grid, const Tfm &t,
                        DevBuf &img, DevBuf &msk, int out_dtype, ResampleJob *jobs, int &nj) {
  ResampleMap mi, mm;
  if (!make_map(grid, src.g, t.M, t.off, mi) || !make_map(grid, mask_g, t.M, t.off, mm)) {
    set_error("singular image geometry");
    return MIRORR_EINVAL;
  }
  const bool same_grid = src.g.size[0] == mask_g.size[0] && src.g.size[1] == mask_g.size[1] &&
                         src.g.size[2] == mask_g.size[2] && memcmp(&mi, &mm, sizeof(mi)) == 0;
  const int ones = c->ones.ptr && mask == c->ones.as<uint8_t>() ? 1 : 0;
  ResampleJob &j = jobs[nj++];
  memset(&j, 0, sizeof(j));
  j.in = static_cast<const float *>(src.img);
  j.out = img.ptr;
  for (int d = 0; d < 3; ++d) { j.in_size[d] = src.g.size[d]; j.out_size[d] = grid.size[d]; }
  memcpy(j.C, mi.C, sizeof(mi.C));
  memcpy(j.e, mi.e, sizeof(mi.e));
  j.out_dtype = out_dtype;
  j.active = 1;
  if (same_grid) {
    j.inm = mask;
    j.outm = msk.as<uint8_t>();
    j.mask_ones = ones;
    return MIRORR_OK;
  }
  ResampleJob &k = jobs[nj++];
  memset(&k, 0, sizeof(k));
  k.inm = mask;
  k.outm = msk.as<uint8_t>();
  for (int d = 0; d < 3; ++d) { k.in_size[d] = mask_g.size[d]; k.out_size[d] = grid.size[d]; }
  memcpy(k.C, mm.C, sizeof(mm.C));
  memcpy(k.e, mm.e, sizeof(mm.e));
  k.active = 1;
  k.mask_ones = ones;
  return MIRORR_OK;
}

// An iteration's launches captured once per pyramid level and replayed for
// its later iterations, and for the same level of later registrations while
// the key is unchanged (float32 storage, no profiling, no per-call printing).
// The key: the level, the middle space and block grid, the parameters baked
// into the launches, and the address and size of every buffer they touch.
std::vector<uint64_t> level_key(mirorr_ctx c, const RegRun &r, const mirorr_geometry &grid,
                                const BmGeom &g, int nj) {
  std::vector<uint64_t> k;
  auto add = [&](uint64_t v) { k.push_back(v); };
  auto buf = [&](const DevBuf &b) {
    add(reinterpret_cast<uint64_t>(b.ptr));
    add(b.bytes);
  };
  add((uint64_t)r.level);
  add((uint64_t)r.p->symmetric);
  add((uint64_t)nj);
  for (int d = 0; d < 3; ++d) add((uint64_t)grid.size[d]);
  uint64_t gb[sizeof(BmGeom) / 8 + 1] = {0};
  memcpy(gb, &g, sizeof(BmGeom));
  for (uint64_t v : gb) add(v);
  uint64_t pb[sizeof(mirorr_bm_params) / 8 + 1] = {0};
  memcpy(pb, &r.p->bm, sizeof(mirorr_bm_params));
  for (uint64_t v : pb) add(v);
  const DevBuf *bufs[] = {&c->bmw.stats, &c->bmw.var, &c->bmw.selected, &c->bmw.select_state,
                          &c->bmw.tiles, &c->bmw.ncc_lists, &c->bmw.ncc_ctl,
                          &c->bmw.ncc_rec, &c->bmw.ncc_bstat, &c->bmw.ncc_pad, &c->bmw.ncc_wand,
                          &c->img_b, &c->img_s, &c->msk_b, &c->msk_s, &c->best, &c->second,
                          &c->match, &c->status, &c->pts_i, &c->pts_m, &c->counts, &c->ncc_count,
                          &c->xl_count, &c->ltsw.state, &c->ltsw.resid, &c->ltsw.partial,
                          &c->ltsw.hist, &c->ltsw.ctrl, &c->ltsw.cand, &c->it_jobs_d};
  for (const DevBuf *b : bufs) buf(*b);
  add(reinterpret_cast<uint64_t>(c->it_jobs.ptr));
  add(reinterpret_cast<uint64_t>(c->it_lts_in.ptr));
  add(reinterpret_cast<uint64_t>(c->it_lts_out.ptr));
  add((uint64_t)c->ltsw.max_ctas);
  add((uint64_t)c->ltsw.spin_limit);
  return k;
}

bool iteration_graphs(const RegRun &r) {
  return r.c->graphs && r.p->storage == MIRORR_DTYPE_F32 && !r.c->timer.on && r.p->verbosity < 2;
}

// Captures issue() on the context's stream into the level's graph, replacing
// the one kept there (the capture always ends).
template <class F>
mirorr_status capture_iteration(mirorr_ctx c, int level, std::vector<uint64_t> key, F issue) {
  auto &g = c->lgraph[level];
  if (g.exec) {
    cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
  }
  g.key.clear();
  MB2_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const mirorr_status rs = issue();
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (rs != MIRORR_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rs;
  }
  if (e != cudaSuccess) {
    set_error("capturing a registration iteration failed: %s", cudaGetErrorString(e));
    return MIRORR_ECUDA;
  }
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g.exec = nullptr;
    set_error("instantiating a registration iteration failed: %s", cudaGetErrorString(e));
    return MIRORR_ECUDA;
  }
  g.key = std::move(key);
  return MIRORR_OK;
}

// After a replayed iteration: the fit's results, as run_lts reports them.
mirorr_status collect_lts(RegRun &r, LtsState &hs, long long *n_used) {
  mirorr_ctx c = r.c;
  unsigned int gave_up = 0;
  int inner = 0;
  MB2_TRY(lts_collect(c->ltsw, c->it_lts_out.ptr, hs, &inner, n_used, &gave_up));
  if (gave_up) {
    bool to = false;
    MB2_TRY(ncc_take_timeout(c->bmw, c->stream, &to));
    set_error("a bounded wait of the block search (a tensor copy or a grid barrier) gave up");
    return MIRORR_ETIMEOUT;
  }
  if (r.stats) {
    r.stats->h2d_bytes += (int64_t)sizeof(LtsState);
    r.stats->d2h_bytes += (int64_t)(sizeof(LtsState) + 2 * sizeof(long long) + 32);
  }
  if (*n_used == 0) {
    set_error("No block matches occurred. Images probably have zero overlap. "
              "Try supplying a better initial transform.");
    return MIRORR_ENOBLOCKS;
  }
  return MIRORR_OK;
}

mirorr_status run_lts(RegRun &r, LtsState &hs, long long nmax, long long *n_used) {
  int inner = 0;
  mirorr_ctx c = r.c;
  unsigned int gave_up = 0;
  const unsigned int *watch = is16(r.p->storage)
                                  ? (c->bm16.ctl.ptr ? c->bm16.ctl.as<unsigned int>() + 2 : nullptr)
                                  : ncc_timeout_flag(c->bmw);
  MB2_TRY(lts_run(c->ltsw, hs, c->pts_i.as<double>(), c->pts_m.as<double>(),
                  c->counts.as<long long>(), nmax, c->stream, &inner, n_used, watch, &gave_up));
  if (gave_up) {
    // a CTA of the search gave up its bounded wait on a tensor copy: that
    // call's scores (and so this fit) cannot be trusted; the registration stops
    bool to = false;
    if (is16(r.p->storage)) MB2_CUDA_TRY(cudaMemsetAsync(c->bm16.ctl.ptr, 0, 16, c->stream));
    else MB2_TRY(ncc_take_timeout(c->bmw, c->stream, &to));
    set_error("a bounded wait of the block search (a tensor copy or a grid barrier) gave up");
    return MIRORR_ETIMEOUT;
  }
  if (r.stats) {
    r.stats->h2d_bytes += (int64_t)sizeof(LtsState);
    r.stats->d2h_bytes += (int64_t)(sizeof(LtsState) + 2 * sizeof(long long) + 32);
  }
  if (c->timer.on) c->timer.harvest();
  if (*n_used == 0) {
    set_error("No block matches occurred. Images probably have zero overlap. "
              "Try supplying a better initial transform.");
    return MIRORR_ENOBLOCKS;
  }
  return MIRORR_OK;
}

mirorr_status ensure_pts(mirorr_ctx c, long long n) {
  MB2_TRY(c->pts_i.ensure(sizeof(double) * 3 * std::max(1LL, n)));
  MB2_TRY(c->pts_m.ensure(sizeof(double) * 3 * std::max(1LL, n)));
  return MIRORR_OK;
}

double param_delta(const double *a, const double *b, int n) {
  double d = 0.0;
  for (int i = 0; i < n; ++i) {
    double e = a[i] - b[i];
    d += e * e;
  }
  return d;
}

void grid_geom(const double *origin, const double *spacing, const int *size,
               const double *direction, mirorr_geometry &g) {
  for (int d = 0; d < 3; ++d) {
    g.origin[d] = origin[d];
    g.spacing[d] = spacing[d];
    g.size[d] = size[d];
  }
  for (int i = 0; i < 9; ++i) g.direction[i] = direction[i];
}

mirorr_status match_into(RegRun &r, const void *base, const uint8_t *bmask, const void *search,
                         const uint8_t *smask, const mirorr_geometry &base_g, double *pts_b,
                         double *pts_m, int count_slot, const long long *offset_dev) {
  mirorr_ctx c = r.c;
  MatchCall mc{base, search, r.p->storage, bmask, smask,
               {base_g.size[0], base_g.size[1], base_g.size[2]}, base_g};
  BmGeom g;
  cudaEvent_t *ev = c->timer.on ? c->timer.take(StageTimer::kPerCall) : nullptr;
  bool xl_ran = false;
  MB2_TRY(run_match(c, r.p->bm, mc, g, c->best, c->second, c->match, c->status, pts_b, pts_m,
                    c->counts.as<long long>() + count_slot, offset_dev, ev, ev ? ev + 5 : nullptr,
                    ev ? c->xl_count.as<unsigned long long>() : nullptr, &xl_ran));
  if (ev) c->timer.ran.push_back(xl_ran ? 1 : 0);
  if (r.stats) r.stats->matcher_calls += 1;
  if (r.p->verbosity >= 2) {
    // per-call routing of the blocks through the search kernels
    unsigned int ctl[8] = {0};
    MB2_CUDA_TRY(cudaMemcpyAsync(ctl, c->bmw.ncc_ctl.ptr, sizeof(ctl), cudaMemcpyDeviceToHost, c->stream));
    MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
    printf("  matcher: %lld blocks, register-blocked %u, masked-window %u, base-mask %u, "
           "refined candidates %u, overflowed %u\n",
           g.nblocks, ctl[3], ctl[4], ctl[0], ctl[2], ctl[1]);
  }
  return MIRORR_OK;
}

mirorr_status classic_level(RegRun &r, const RegImage &fl, const RegImage &ml, Tfm &tfm) {
  mirorr_ctx c = r.c;
  const mirorr_reg_params &p = *r.p;
  double cf[3], cm[3], origin[3], spacing[3];
  int size[3];
  center_of(fl.g, cf);
  center_of(ml.g, cm);
  for (int d = 0; d < 3; ++d) {
    origin[d] = cm[d] + ((fl.g.origin[d] - cf[d]) + (ml.g.origin[d] - cm[d])) / 2.0;
    spacing[d] = (fl.g.spacing[d] + ml.g.spacing[d]) / 2.0;
    size[d] = (int)(((double)fl.g.size[d] + (double)ml.g.size[d] + 0.5) / 2.0);
  }
  mirorr_geometry grid_f, grid_m;
  grid_geom(origin, spacing, size, fl.g.direction, grid_f);
  grid_geom(origin, spacing, size, ml.g.direction, grid_m);
  Tfm ident;
  tfm_identity(ident, KIND_AFFINE);
  MB2_TRY(resample_into(c, ml, r.mmask, r.mmask_g, grid_m, ident, c->img_b, c->msk_b, p.storage));
  BmGeom g;
  if (!bm_geometry(size, (int)p.bm.block_width, (int)p.bm.block_gap, (int)p.bm.nhood_gap,
                   (int)p.bm.nhood_width, g)) {
    set_error("middle-space image smaller than one block");
    return MIRORR_EINVAL;
  }
  MB2_TRY(ensure_pts(c, g.nblocks));
  double last[12], cur[12];
  tfm_params(tfm, last);
  int np = tfm_nparams(tfm);
  int it = 0;
  const bool graphs = iteration_graphs(r) && r.level < 16;
  for (; it < std::abs(p.iterations); ++it) {
    LtsState hs;
    memset(&hs, 0, sizeof(hs));
    hs.kind = tfm.kind;
    hs.symmetric = 0;
    hs.lts_keep = p.lts_keep;
    hs.tfm = tfm;
    long long used = 0;
    // the level's graph: kept from an earlier iteration or registration when
    // its key matches; else captured at the second iteration (the first one
    // runs directly and sizes every buffer)
    int nj = 0;
    std::vector<uint64_t> key;
    bool use_graph = false;
    if (graphs) {
      ResampleJob *jobs = c->it_jobs.as<ResampleJob>();
      MB2_TRY(make_jobs(c, fl, r.fmask, r.fmask_g, grid_f, tfm, c->img_s, c->msk_s, p.storage, jobs, nj));
      key = level_key(c, r, grid_f, g, nj);
      use_graph = (c->lgraph[r.level].exec && c->lgraph[r.level].key == key) || it > 0;
    }
    if (use_graph) {
      lts_begin(hs);
      memcpy(c->it_lts_in.ptr, &hs, sizeof(hs));
      if (!c->lgraph[r.level].exec || c->lgraph[r.level].key != key) {
        const int64_t calls0 = r.stats ? r.stats->matcher_calls : 0;
        MB2_TRY(capture_iteration(c, r.level, key, [&]() -> mirorr_status {
          MB2_CUDA_TRY(cudaMemcpyAsync(c->it_jobs_d.ptr, c->it_jobs.ptr, sizeof(ResampleJob) * nj,
                                       cudaMemcpyHostToDevice, c->stream));
          MB2_TRY(launch_resample_batch(c->it_jobs_d.as<ResampleJob>(), nj, vox(grid_f.size), c->stream));
          MB2_CUDA_TRY(cudaMemsetAsync(c->counts.ptr, 0, 4 * sizeof(long long), c->stream));
          MB2_TRY(match_into(r, c->img_b.ptr, c->msk_b.as<uint8_t>(), c->img_s.ptr,
                             c->msk_s.as<uint8_t>(), grid_m, c->pts_i.as<double>(),
                             c->pts_m.as<double>(), 0, nullptr));
          return lts_issue(c->ltsw, c->it_lts_in.as<LtsState>(), c->pts_i.as<double>(),
                           c->pts_m.as<double>(), c->counts.as<long long>(), g.nblocks, c->stream,
                           c->it_lts_out.ptr, ncc_timeout_flag(c->bmw));
        }));
        if (r.stats) r.stats->matcher_calls = calls0;
      }
      MB2_CUDA_TRY(cudaGraphLaunch(c->lgraph[r.level].exec, c->stream));
      MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
      if (r.stats) r.stats->matcher_calls += 1;
      MB2_TRY(collect_lts(r, hs, &used));
    } else {
      MB2_TRY(resample_into(c, fl, r.fmask, r.fmask_g, grid_f, tfm, c->img_s, c->msk_s, p.storage));
      MB2_CUDA_TRY(cudaMemsetAsync(c->counts.ptr, 0, 4 * sizeof(long long), c->stream));
      MB2_TRY(match_into(r, c->img_b.ptr, c->msk_b.as<uint8_t>(), c->img_s.ptr,
                         c->msk_s.as<uint8_t>(), grid_m, c->pts_i.as<double>(),
                         c->pts_m.as<double>(), 0, nullptr));
      MB2_TRY(run_lts(r, hs, g.nblocks, &used));
    }
    tfm = hs.tfm;
    tfm_params(tfm, cur);
    double d = param_delta(last, cur, np);
    for (int i = 0; i < 12; ++i) last[i] = cur[i];
    if (p.verbosity >= 1)
      printf("level %d iteration %d: blocks %lld, delta %.6g\n", r.level, it + 1, used, d);
    if (d < 1e-3) { ++it; break; }
  }
  if (r.stats && r.level < 16) r.stats->iterations_run[r.level] = it;
  return MIRORR_OK;
}

mirorr_status symmetric_level(RegRun &r, const RegImage &fl, const RegImage &ml, Tfm &tfm) {
  mirorr_ctx c = r.c;
  const mirorr_reg_params &p = *r.p;
  double cf[3], cm[3], origin[3], spacing[3];
  int size[3];
  center_of(fl.g, cf);
  center_of(ml.g, cm);
  for (int d = 0; d < 3; ++d) {
    origin[d] = ((fl.g.origin[d] - cf[d]) + (ml.g.origin[d] - cm[d])) / 2.0;
    spacing[d] = (fl.g.spacing[d] + ml.g.spacing[d]) / 2.0;
    size[d] = (int)(((double)fl.g.size[d] + (double)ml.g.size[d] + 0.5) / 2.0);
  }
  mirorr_geometry grid_f, grid_m;
  grid_geom(origin, spacing, size, fl.g.direction, grid_f);
  grid_geom(origin, spacing, size, ml.g.direction, grid_m);
  double initial_center[3] = {tfm.c[0], tfm.c[1], tfm.c[2]};
  tfm_center_to_origin(tfm);
  Tfm fixed_tr, moving_tr, ifixed;
  tfm_identity(fixed_tr, KIND_RIGID);
  tfm_identity(moving_tr, KIND_RIGID);
  double pf[6] = {0, 0, 0, cf[0], cf[1], cf[2]}, pm[6] = {0, 0, 0, cm[0], cm[1], cm[2]};
  tfm_set_params(fixed_tr, pf);
  tfm_set_params(moving_tr, pm);
  tfm_inverse(fixed_tr, ifixed);
  tfm_compose(tfm, ifixed, false);
  tfm_compose(tfm, moving_tr, true);
  Tfm t12f, t12b;
  half_space(tfm, t12f, t12b);
  BmGeom g;
  if (!bm_geometry(size, (int)p.bm.block_width, (int)p.bm.block_gap, (int)p.bm.nhood_gap,
                   (int)p.bm.nhood_width, g)) {
    set_error("middle-space image smaller than one block");
    return MIRORR_EINVAL;
  }
  MB2_TRY(ensure_pts(c, 2 * g.nblocks));
  double last[12], cur[12], prm[12];
  tfm_params(tfm, last);
  int np = tfm_nparams(tfm);
  auto centered = [&](Tfm &cF, Tfm &cB) {
    tfm_identity(cF, tfm.kind);
    tfm_identity(cB, tfm.kind);
    tfm_params(t12f, prm);
    tfm_set_params(cF, prm);
    tfm_compose(cF, fixed_tr, false);
    tfm_params(t12b, prm);
    tfm_set_params(cB, prm);
    tfm_compose(cB, moving_tr, false);
  };
  int it = 0;
  const bool graphs = iteration_graphs(r) && r.level < 16;
  for (; it < std::abs(p.iterations); ++it) {
    Tfm cF, cB;
    centered(cF, cB);
    double *pi = c->pts_i.as<double>(), *pmv = c->pts_m.as<double>();
    LtsState hs;
    memset(&hs, 0, sizeof(hs));
    hs.kind = tfm.kind;
    hs.symmetric = 1;
    hs.lts_keep = p.lts_keep;
    hs.tfm = tfm;
    hs.t12f = t12f;
    hs.t12b = t12b;
    long long used = 0;
    // the level's graph: kept from an earlier iteration or registration when
    // its key matches; else captured at the second iteration (the first one
    // runs directly and sizes every buffer)
    int nj = 0;
    std::vector<uint64_t> key;
    bool use_graph = false;
    if (graphs) {
      ResampleJob *jobs = c->it_jobs.as<ResampleJob>();
      MB2_TRY(make_jobs(c, ml, r.mmask, r.mmask_g, grid_m, cB, c->img_b, c->msk_b, p.storage, jobs, nj));
      MB2_TRY(make_jobs(c, fl, r.fmask, r.fmask_g, grid_f, cF, c->img_s, c->msk_s, p.storage, jobs, nj));
      key = level_key(c, r, grid_f, g, nj);
      use_graph = (c->lgraph[r.level].exec && c->lgraph[r.level].key == key) || it > 0;
    }
    if (use_graph) {
      lts_begin(hs);
      memcpy(c->it_lts_in.ptr, &hs, sizeof(hs));
      if (!c->lgraph[r.level].exec || c->lgraph[r.level].key != key) {
        const int64_t calls0 = r.stats ? r.stats->matcher_calls : 0;
        MB2_TRY(capture_iteration(c, r.level, key, [&]() -> mirorr_status {
          MB2_CUDA_TRY(cudaMemcpyAsync(c->it_jobs_d.ptr, c->it_jobs.ptr, sizeof(ResampleJob) * nj,
                                       cudaMemcpyHostToDevice, c->stream));
          MB2_TRY(launch_resample_batch(c->it_jobs_d.as<ResampleJob>(), nj, vox(grid_f.size), c->stream));
          MB2_CUDA_TRY(cudaMemsetAsync(c->counts.ptr, 0, 4 * sizeof(long long), c->stream));
          MB2_TRY(match_into(r, c->img_b.ptr, c->msk_b.as<uint8_t>(), c->img_s.ptr,
                             c->msk_s.as<uint8_t>(), grid_m, pi, pmv, 0, nullptr));
          MB2_TRY(match_into(r, c->img_s.ptr, c->msk_s.as<uint8_t>(), c->img_b.ptr,
                             c->msk_b.as<uint8_t>(), grid_f, pmv, pi, 1, c->counts.as<long long>()));
          return lts_issue(c->ltsw, c->it_lts_in.as<LtsState>(), pi, pmv, c->counts.as<long long>(),
                           2 * g.nblocks, c->stream, c->it_lts_out.ptr, ncc_timeout_flag(c->bmw));
        }));
        if (r.stats) r.stats->matcher_calls = calls0;
      }
      MB2_CUDA_TRY(cudaGraphLaunch(c->lgraph[r.level].exec, c->stream));
      MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
      if (r.stats) r.stats->matcher_calls += 2;
      MB2_TRY(collect_lts(r, hs, &used));
    } else {
      MB2_TRY(resample_into(c, ml, r.mmask, r.mmask_g, grid_m, cB, c->img_b, c->msk_b, p.storage));
      MB2_TRY(resample_into(c, fl, r.fmask, r.fmask_g, grid_f, cF, c->img_s, c->msk_s, p.storage));
      MB2_CUDA_TRY(cudaMemsetAsync(c->counts.ptr, 0, 4 * sizeof(long long), c->stream));
      // forward: base = moving, search = fixed
      MB2_TRY(match_into(r, c->img_b.ptr, c->msk_b.as<uint8_t>(), c->img_s.ptr,
                         c->msk_s.as<uint8_t>(), grid_m, pi, pmv, 0, nullptr));
      // swapped: base = fixed, search = moving; its lists are appended with
      // roles reversed (itkSymMirorrRegistrationMethod.txx:595-602)
      MB2_TRY(match_into(r, c->img_s.ptr, c->msk_s.as<uint8_t>(), c->img_b.ptr,
                         c->msk_b.as<uint8_t>(), grid_f, pmv, pi, 1, c->counts.as<long long>()));
      MB2_TRY(run_lts(r, hs, 2 * g.nblocks, &used));
    }
    tfm = hs.tfm;
    t12f = hs.t12f;
    t12b = hs.t12b;
    tfm_params(tfm, cur);
    double d = param_delta(last, cur, np);
    for (int i = 0; i < 12; ++i) last[i] = cur[i];
    if (p.verbosity >= 1)
      printf("level %d iteration %d: blocks %lld, delta %.6g\n", r.level, it + 1, used, d);
    if (d < 1e-3) { ++it; break; }
  }
  if (r.stats && r.level < 16) r.stats->iterations_run[r.level] = it;
  Tfm cF, cB, ib;
  centered(cF, cB);
  tfm_inverse(cB, ib);
  tfm_identity(tfm, tfm.kind);
  tfm_compose(tfm, ib, true);
  tfm_compose(tfm, cF, false);
  tfm_update_center(tfm, initial_center);
  return MIRORR_OK;
}

mirorr_status register_impl(mirorr_ctx c, const mirorr_geometry *fg, const void *fixed,
                            const uint8_t *fmask, const mirorr_geometry *mg, const void *moving,
                            const uint8_t *mmask, const mirorr_reg_params *p,
                            const mirorr_transform *init, mirorr_transform *result,
                            mirorr_reg_stats *stats) {
  if (!c || !fg || !mg || !fixed || !moving || !p || !result) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  if (!valid_geom(fg) || !valid_geom(mg)) {
    set_error("invalid image geometry");
    return MIRORR_EINVAL;
  }
  if (p->kind != KIND_RIGID && p->kind != KIND_AFFINE) {
    set_error("transform kind must be 0 (rigid) or 1 (affine)");
    return MIRORR_EINVAL;
  }
  MB2_TRY(check_bm_params(p->bm));
  if (p->storage != MIRORR_DTYPE_F32 && !is16(p->storage)) {
    set_error("storage must be MIRORR_DTYPE_F32, _BF16 or _F16 (got %d)", p->storage);
    return MIRORR_EINVAL;
  }
  if (!(p->lts_keep > 0.0 && p->lts_keep <= 1.0)) {
    set_error("lts_keep must lie in (0, 1]");
    return MIRORR_EINVAL;
  }
  auto t0 = std::chrono::steady_clock::now();
  mirorr_reg_params pp = *p;
  if (pp.iterations == 0) pp.iterations = 5;
  if (pp.min_length <= 0) pp.min_length = 32;
  MB2_TRY(c->counts.ensure(4 * sizeof(long long)));
  MB2_TRY(c->ncc_count.ensure(sizeof(unsigned long long)));
  MB2_TRY(c->it_jobs.ensure(sizeof(ResampleJob) * 4));
  MB2_TRY(c->it_jobs_d.ensure(sizeof(ResampleJob) * 4));
  MB2_TRY(c->it_lts_in.ensure(sizeof(LtsState)));
  MB2_TRY(c->it_lts_out.ensure(lts_out_bytes()));
  MB2_CUDA_TRY(cudaMemsetAsync(c->ncc_count.ptr, 0, sizeof(unsigned long long), c->stream));
  if (stats) memset(stats, 0, sizeof(*stats));
  long long nmax = std::max(vox(fg->size), vox(mg->size));
  if (!fmask || !mmask) MB2_TRY(ensure_ones(c, nmax));
  RegRun r{c, &pp, fmask ? fmask : c->ones.as<uint8_t>(), mmask ? mmask : c->ones.as<uint8_t>(),
           *fg, *mg, stats, 0};
  int sm[16][3], sf[16][3];
  int nl = pyramid_schedule(*fg, *mg, pp.min_length, pp.levels, sm, sf);
  if (pp.last_level > 0 && pp.last_level < nl) nl = pp.last_level;
  else if (pp.last_level < 0) nl = std::max(1, nl + pp.last_level);
  Tfm tfm;
  if (init) {
    if (!from_public(*init, tfm) || init->kind != pp.kind) {
      set_error("initial transform kind does not match the requested kind");
      return MIRORR_EINVAL;
    }
  } else {
    double cfix[3], cmov[3], tr[3];
    center_of(*fg, cfix);
    center_of(*mg, cmov);
    tfm_identity(tfm, pp.kind);
    tfm_set_center(tfm, cmov);
    for (int d = 0; d < 3; ++d) tr[d] = cfix[d] - cmov[d];
    tfm_set_translation(tfm, tr);
  }
  double params[12];
  tfm_params(tfm, params);
  for (int lev = 0; lev < nl; ++lev) {
    RegImage fl, ml;
    MB2_TRY(make_level(c, *fg, fixed, pp.storage, sf[lev], fl.g, c->lvl_f, &fl.img, &fl.dtype));
    MB2_TRY(make_level(c, *mg, moving, pp.storage, sm[lev], ml.g, c->lvl_m, &ml.img, &ml.dtype));
    tfm_set_params(tfm, params);
    r.level = lev;
    if (pp.symmetric) MB2_TRY(symmetric_level(r, fl, ml, tfm));
    else MB2_TRY(classic_level(r, fl, ml, tfm));
    tfm_params(tfm, params);
  }
  tfm_set_params(tfm, params);
  {
    bool to = false, to16 = false;
    MB2_TRY(ncc_take_timeout(c->bmw, c->stream, &to));
    MB2_TRY(match16_take_timeout(c->bm16, c->stream, &to16));
    if (to || to16) {
      set_error("a bounded wait of the block search (a tensor copy or a grid barrier) gave up");
      return MIRORR_ETIMEOUT;
    }
  }
  to_public(tfm, *result);
  if (stats) {
    stats->levels_run = nl;
    unsigned long long cnt = 0;
    MB2_CUDA_TRY(cudaMemcpyAsync(&cnt, c->ncc_count.ptr, sizeof(cnt), cudaMemcpyDeviceToHost,
                                 c->stream));
    MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
    stats->block_ncc_evaluated = (int64_t)cnt;
    stats->d2h_bytes += (int64_t)sizeof(cnt);
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return MIRORR_OK;
}

mirorr_status upload(mirorr_ctx c, DevBuf &b, const void *host, size_t bytes) {
  MB2_TRY(b.ensure(bytes));
  MB2_CUDA_TRY(cudaMemcpyAsync(b.ptr, host, bytes, cudaMemcpyHostToDevice, c->stream));
  return MIRORR_OK;
}

}  // namespace

// ============================================================================
extern "C" {

const char *mirorr_last_error(void) { return mb2::get_error(); }
int32_t mirorr_abi_version(void) { return MIRORR_ABI_VERSION; }

mirorr_status mirorr_ctx_create(int32_t device, mirorr_ctx *out) {
  if (!out) { set_error("null argument"); return MIRORR_EINVAL; }
  *out = nullptr;
  MB2_TRY(check_device(device));
  MB2_CUDA_TRY(cudaSetDevice(device));
  mirorr_ctx c = new (std::nothrow) mirorr_ctx_s;
  if (!c) { set_error("out of host memory"); return MIRORR_ENOMEM; }
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    set_error("cudaStreamCreate failed: %s", cudaGetErrorString(e));
    return MIRORR_ECUDA;
  }
  c->launches0 = g_launches;
  mirorr_status s = c->counts.ensure(4 * sizeof(long long));
  if (s == MIRORR_OK) s = c->ncc_count.ensure(sizeof(unsigned long long));
  if (s != MIRORR_OK) { mirorr_ctx_destroy(c); return s; }
  *out = c;
  return MIRORR_OK;
}

mirorr_status mirorr_ctx_destroy(mirorr_ctx c) {
  if (!c) return MIRORR_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DevBuf *bufs[] = {&c->bmw.stats, &c->bmw.var, &c->bmw.selected, &c->bmw.select_state,
                    &c->bmw.tiles, &c->bmw.ncc_lists, &c->bmw.ncc_ctl, &c->bmw.ncc_rec, &c->bmw.ncc_bstat, &c->bmw.ncc_pad, &c->bmw.ncc_wand, &c->ltsw.state, &c->ltsw.resid, &c->xl_count,
                    &c->ltsw.partial, &c->ltsw.hist, &c->ltsw.ctrl, &c->ltsw.cand, &c->counts,
                    &c->ncc_count, &c->ones, &c->lvl_f, &c->lvl_m, &c->tmp_a, &c->tmp_b,
                    &c->weights, &c->img_b, &c->img_s, &c->msk_b, &c->msk_s, &c->best,
                    &c->second, &c->match, &c->status, &c->pts_i, &c->pts_m, &c->up_f,
                    &c->up_m, &c->up_fm, &c->up_mm, &c->bm16.stats, &c->bm16.wand,
                    &c->bm16.prep, &c->bm16.xs, &c->bm16.ctl, &c->bm16.fb_list,
                    &c->bm16.chunked, &c->bm16.calls, &c->it_jobs_d};
  for (DevBuf *b : bufs) b->release();
  HostBuf *hbufs[] = {&c->it_jobs, &c->it_lts_in, &c->it_lts_out, &c->ltsw.out};
  for (HostBuf *b : hbufs) b->release();
  for (auto &lg : c->lgraph)
    if (lg.exec) cudaGraphExecDestroy(lg.exec);
  c->timer.release();
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return MIRORR_OK;
}

int64_t mirorr_ctx_kernel_launches(mirorr_ctx c) { return c ? g_launches - c->launches0 : g_launches; }

void *mirorr_ctx_stream(mirorr_ctx c) { return c ? (void *)c->stream : nullptr; }

mirorr_status mirorr_ctx_set_graphs(mirorr_ctx c, int32_t on) {
  if (!c) { set_error("null argument"); return MIRORR_EINVAL; }
  c->graphs = on != 0;
  return MIRORR_OK;
}

mirorr_status mirorr_ctx_set_profiling(mirorr_ctx c, int32_t on) {
  if (!c) { set_error("null argument"); return MIRORR_EINVAL; }
  if (on && !c->xl_count.ptr) {
    MB2_CUDA_TRY(cudaSetDevice(c->device));
    MB2_TRY(c->xl_count.ensure(sizeof(unsigned long long)));
    MB2_CUDA_TRY(cudaMemsetAsync(c->xl_count.ptr, 0, sizeof(unsigned long long), c->stream));
  }
  c->timer.on = on != 0;
  return MIRORR_OK;
}

mirorr_status mirorr_ctx_search_kernel_times(mirorr_ctx c, double *ms, int64_t *launches,
                                             int64_t *candidates) {
  if (!c || !ms) { set_error("null argument"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->timer.harvest();
  unsigned long long n = 0;
  if (c->xl_count.ptr) {
    MB2_CUDA_TRY(cudaMemcpy(&n, c->xl_count.ptr, sizeof(n), cudaMemcpyDeviceToHost));
    MB2_CUDA_TRY(cudaMemset(c->xl_count.ptr, 0, sizeof(n)));
  }
  *ms = c->timer.search_ms;
  if (launches) *launches = c->timer.search_calls;
  if (candidates) *candidates = (int64_t)n;
  c->timer.search_ms = 0.0;
  c->timer.search_calls = 0;
  return MIRORR_OK;
}

mirorr_status mirorr_ctx_resample_times(mirorr_ctx c, double *ms, int64_t *passes,
                                        int64_t *voxels) {
  if (!c || !ms) { set_error("null argument"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->timer.harvest();
  *ms = c->timer.resample_ms;
  if (passes) *passes = c->timer.resample_passes;
  if (voxels) *voxels = c->timer.resample_voxels;
  c->timer.resample_ms = 0.0;
  c->timer.resample_passes = 0;
  c->timer.resample_voxels = 0;
  return MIRORR_OK;
}

mirorr_status mirorr_ctx_set_wait_limit(mirorr_ctx c, int64_t polls) {
  if (!c || polls < 0) { set_error("null context or negative limit"); return MIRORR_EINVAL; }
  c->ltsw.spin_limit = polls;
  return MIRORR_OK;
}

mirorr_status mirorr_ctx_stage_times(mirorr_ctx c, double ms[4], int64_t *calls) {
  if (!c || !ms) { set_error("null argument"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->timer.harvest();
  for (int i = 0; i < 4; ++i) { ms[i] = c->timer.ms[i]; c->timer.ms[i] = 0.0; }
  if (calls) *calls = c->timer.calls;
  c->timer.calls = 0;
  return MIRORR_OK;
}

// ---- block matcher -----------------------------------------------------------
mirorr_status mirorr_bm_default_params(mirorr_bm_params *p) {
  if (!p) { set_error("null argument"); return MIRORR_EINVAL; }
  p->block_width = 4;
  p->block_gap = 1;
  p->nhood_gap = 2;
  p->nhood_width = 5;
  p->portion_matches_kept = 0.5;
  p->block_keep = 1.0;
  p->verbosity = 0;
  return MIRORR_OK;
}

mirorr_status mirorr_bm_create(mirorr_ctx c, mirorr_matcher *out) {
  if (!c || !out) { set_error("null argument"); return MIRORR_EINVAL; }
  mirorr_matcher m = new (std::nothrow) mirorr_matcher_s;
  if (!m) { set_error("out of host memory"); return MIRORR_ENOMEM; }
  m->ctx = c;
  mirorr_bm_default_params(&m->p);
  for (auto &e : m->ev) {
    if (cudaEventCreate(&e) != cudaSuccess) {
      set_error("cudaEventCreate failed");
      mirorr_bm_destroy(m);
      return MIRORR_ECUDA;
    }
  }
  *out = m;
  return MIRORR_OK;
}

mirorr_status mirorr_bm_destroy(mirorr_matcher m) {
  if (!m) return MIRORR_OK;
  for (auto &e : m->ev)
    if (e) cudaEventDestroy(e);
  DevBuf *bufs[] = {&m->base.own_img, &m->base.own_mask, &m->search.own_img,
                    &m->search.own_mask, &m->best, &m->second, &m->match, &m->status,
                    &m->pts_b, &m->pts_m};
  for (DevBuf *b : bufs) b->release();
  delete m;
  return MIRORR_OK;
}

mirorr_status mirorr_bm_set_params(mirorr_matcher m, const mirorr_bm_params *p) {
  if (!m || !p) { set_error("null argument"); return MIRORR_EINVAL; }
  mirorr_bm_params q = *p;
  if (q.portion_matches_kept == 0.0) q.portion_matches_kept = 0.5;
  MB2_TRY(check_bm_params(q));
  m->p = q;
  return MIRORR_OK;
}

mirorr_status mirorr_bm_set_metric(mirorr_matcher m, const char *name) {
  if (!m || !name) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!strcmp(name, "nc") || !strcmp(name, "normalized_correlation")) return MIRORR_OK;
  set_error("block metric '%s' is not available on this path (only normalized_correlation)", name);
  return MIRORR_EINVAL;
}

// Sets an image.  host: float32 copied to the device; dev32: a float32 device
// buffer; dev16: a device buffer already in the 16-bit storage type.  With
// 16-bit storage, float32 input is converted (round to nearest) into a copy
// the matcher owns; with float32 storage a device buffer is borrowed.
enum class ImgSrc { host, dev32, dev16 };

static mirorr_status set_image(mirorr_matcher m, Vol &v, const mirorr_geometry *g,
                               const void *p, ImgSrc src) {
  if (!m || !g || !p) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!valid_geom(g)) { set_error("invalid geometry"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(m->ctx->device));
  const long long n = vox(g->size);
  if (src == ImgSrc::dev16) {
    if (!is16(m->storage)) {
      set_error("16-bit images need BF16 or F16 storage (mirorr_bm_set_storage)");
      return MIRORR_ESTATE;
    }
    v.img = p;
  } else if (!is16(m->storage)) {
    if (src == ImgSrc::host) {
      MB2_TRY(upload(m->ctx, v.own_img, p, sizeof(float) * n));
      v.img = v.own_img.ptr;
    } else {
      v.img = p;
    }
  } else {
    const float *f32 = static_cast<const float *>(p);
    if (src == ImgSrc::host) {
      MB2_TRY(upload(m->ctx, m->ctx->up_f, p, sizeof(float) * n));
      f32 = m->ctx->up_f.as<float>();
    }
    MB2_TRY(v.own_img.ensure(2 * n));
    MB2_TRY(launch_to16(f32, v.own_img.ptr, n, m->storage, m->ctx->stream));
    v.img = v.own_img.ptr;
  }
  if (v.has && vox(v.geom.size) != n && v.has_mask) {
    v.has_mask = false;  // a mask of the old size no longer applies
    v.mask = nullptr;
  }
  v.geom = *g;
  v.has = true;
  m->has_results = false;
  return MIRORR_OK;
}

static mirorr_status set_mask(mirorr_matcher m, Vol &v, const uint8_t *p, bool host) {
  if (!m) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!p) {
    v.has_mask = false;
    v.mask = nullptr;
    return MIRORR_OK;
  }
  if (!v.has) { set_error("set the image before its mask"); return MIRORR_ESTATE; }
  MB2_CUDA_TRY(cudaSetDevice(m->ctx->device));
  if (host) {
    MB2_TRY(upload(m->ctx, v.own_mask, p, vox(v.geom.size)));
    v.mask = v.own_mask.as<uint8_t>();
  } else {
    v.mask = p;
  }
  v.has_mask = true;
  m->has_results = false;
  return MIRORR_OK;
}

mirorr_status mirorr_bm_set_base_image(mirorr_matcher m, const mirorr_geometry *g, const float *h) {
  return m ? set_image(m, m->base, g, h, ImgSrc::host) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_search_image(mirorr_matcher m, const mirorr_geometry *g, const float *h) {
  return m ? set_image(m, m->search, g, h, ImgSrc::host) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_base_image_device(mirorr_matcher m, const mirorr_geometry *g,
                                              const float *d) {
  return m ? set_image(m, m->base, g, d, ImgSrc::dev32) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_search_image_device(mirorr_matcher m, const mirorr_geometry *g,
                                                const float *d) {
  return m ? set_image(m, m->search, g, d, ImgSrc::dev32) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_storage(mirorr_matcher m, int32_t dtype) {
  if (!m) { set_error("null argument"); return MIRORR_EINVAL; }
  if (dtype != MIRORR_DTYPE_F32 && !is16(dtype)) {
    set_error("storage must be MIRORR_DTYPE_F32, _BF16 or _F16 (got %d)", dtype);
    return MIRORR_EINVAL;
  }
  if (dtype != m->storage) {
    // images of the old type no longer apply
    m->base.has = m->search.has = false;
    m->base.img = m->search.img = nullptr;
    m->has_results = false;
  }
  m->storage = dtype;
  return MIRORR_OK;
}
mirorr_status mirorr_bm_set_base_image_device16(mirorr_matcher m, const mirorr_geometry *g,
                                                const void *d) {
  return m ? set_image(m, m->base, g, d, ImgSrc::dev16) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_search_image_device16(mirorr_matcher m, const mirorr_geometry *g,
                                                  const void *d) {
  return m ? set_image(m, m->search, g, d, ImgSrc::dev16) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_base_mask(mirorr_matcher m, const uint8_t *h) {
  return m ? set_mask(m, m->base, h, true) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_search_mask(mirorr_matcher m, const uint8_t *h) {
  return m ? set_mask(m, m->search, h, true) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_base_mask_device(mirorr_matcher m, const uint8_t *d) {
  return m ? set_mask(m, m->base, d, false) : MIRORR_EINVAL;
}
mirorr_status mirorr_bm_set_search_mask_device(mirorr_matcher m, const uint8_t *d) {
  return m ? set_mask(m, m->search, d, false) : MIRORR_EINVAL;
}

mirorr_status mirorr_bm_swap_image_order(mirorr_matcher m) {
  if (!m) { set_error("null argument"); return MIRORR_EINVAL; }
  std::swap(m->base.img, m->search.img);
  std::swap(m->base.mask, m->search.mask);
  std::swap(m->base.has, m->search.has);
  std::swap(m->base.has_mask, m->search.has_mask);
  std::swap(m->base.geom, m->search.geom);
  std::swap(m->base.own_img, m->search.own_img);
  std::swap(m->base.own_mask, m->search.own_mask);
  m->has_results = false;
  return MIRORR_OK;
}

mirorr_status mirorr_bm_grid(mirorr_matcher m, int32_t nblocks[3], int32_t start[3]) {
  if (!m || !nblocks || !start) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!m->base.has) { set_error("base image not set"); return MIRORR_ESTATE; }
  BmGeom g;
  if (!bm_geometry(m->base.geom.size, (int)m->p.block_width, (int)m->p.block_gap,
                   (int)m->p.nhood_gap, (int)m->p.nhood_width, g)) {
    set_error("image smaller than one block");
    return MIRORR_EINVAL;
  }
  for (int d = 0; d < 3; ++d) { nblocks[d] = g.nb[d]; start[d] = g.st[d]; }
  return MIRORR_OK;
}

mirorr_status mirorr_bm_get_offsets(mirorr_matcher m, size_t capacity, double *bp, double *mp,
                                    size_t *n_out) {
  if (!m || !n_out) { set_error("null argument"); return MIRORR_EINVAL; }
  *n_out = 0;
  if (!m->base.has || !m->search.has) {
    set_error("base and search images must be set before GetOffsets");
    return MIRORR_ESTATE;
  }
  for (int d = 0; d < 3; ++d)
    if (m->base.geom.size[d] != m->search.geom.size[d]) {
      set_error("base and search images must share one grid size");
      return MIRORR_EINVAL;
    }
  mirorr_ctx c = m->ctx;
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  long long nv = vox(m->base.geom.size);
  if (!m->base.has_mask || !m->search.has_mask) MB2_TRY(ensure_ones(c, nv));
  const uint8_t *bmask = m->base.has_mask ? m->base.mask : c->ones.as<uint8_t>();
  const uint8_t *smask = m->search.has_mask ? m->search.mask : c->ones.as<uint8_t>();
  BmGeom g;
  if (!bm_geometry(m->base.geom.size, (int)m->p.block_width, (int)m->p.block_gap,
                   (int)m->p.nhood_gap, (int)m->p.nhood_width, g)) {
    set_error("image smaller than one block");
    return MIRORR_EINVAL;
  }
  MB2_TRY(m->pts_b.ensure(sizeof(double) * 3 * g.nblocks));
  MB2_TRY(m->pts_m.ensure(sizeof(double) * 3 * g.nblocks));
  MB2_CUDA_TRY(cudaMemsetAsync(c->counts.ptr, 0, 4 * sizeof(long long), c->stream));
  MatchCall mc{m->base.img, m->search.img, m->storage, bmask, smask,
               {m->base.geom.size[0], m->base.geom.size[1], m->base.geom.size[2]},
               m->base.geom};
  MB2_TRY(run_match(c, m->p, mc, g, m->best, m->second, m->match, m->status,
                    m->pts_b.as<double>(), m->pts_m.as<double>(), c->counts.as<long long>(),
                    nullptr, m->ev));
  long long kept = 0;
  MB2_CUDA_TRY(cudaMemcpyAsync(&kept, c->counts.ptr, sizeof(kept), cudaMemcpyDeviceToHost,
                               c->stream));
  MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int s = 0; s < 4; ++s) cudaEventElapsedTime(&m->timings[s], m->ev[s], m->ev[s + 1]);
  {
    bool to = false, to_sel = false;
    // the variance selection reports through the FP32 search's flag
    if (is16(m->storage)) MB2_TRY(match16_take_timeout(c->bm16, c->stream, &to));
    MB2_TRY(ncc_take_timeout(c->bmw, c->stream, &to_sel));
    if (to || to_sel) {
      set_error("a bounded wait of the block search (a tensor copy or a grid barrier) gave up");
      return MIRORR_ETIMEOUT;
    }
  }
  m->last = g;
  m->kept = kept;
  m->has_results = true;
  *n_out = (size_t)kept;
  if (kept == 0) {
    set_error("No block matches occurred. Images probably have zero overlap. "
              "Try supplying a better initial transform.");
    return MIRORR_ENOBLOCKS;
  }
  if ((size_t)kept > capacity) {
    set_error("output capacity %zu < %lld kept blocks", capacity, kept);
    return MIRORR_ERANGE;
  }
  if (bp)
    MB2_CUDA_TRY(cudaMemcpy(bp, m->pts_b.ptr, sizeof(double) * 3 * kept, cudaMemcpyDeviceToHost));
  if (mp)
    MB2_CUDA_TRY(cudaMemcpy(mp, m->pts_m.ptr, sizeof(double) * 3 * kept, cudaMemcpyDeviceToHost));
  return MIRORR_OK;
}

mirorr_status mirorr_bm_block_results(mirorr_matcher m, size_t capacity, int32_t *match_index,
                                      float *best, float *second, uint8_t *status,
                                      size_t *n_blocks) {
  if (!m || !n_blocks) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!m->has_results) { set_error("no results: call GetOffsets first"); return MIRORR_ESTATE; }
  long long n = m->last.nblocks;
  *n_blocks = (size_t)n;
  if ((size_t)n > capacity) { set_error("capacity too small"); return MIRORR_ERANGE; }
  MB2_CUDA_TRY(cudaSetDevice(m->ctx->device));
  if (match_index) {
    std::vector<int32_t> lin(n);
    MB2_CUDA_TRY(cudaMemcpy(lin.data(), m->match.ptr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    const int nx = m->last.size[0], ny = m->last.size[1];
    for (long long b = 0; b < n; ++b) {
      int v = lin[b];
      match_index[3 * b] = v % nx;
      match_index[3 * b + 1] = (v / nx) % ny;
      match_index[3 * b + 2] = v / (nx * ny);
    }
  }
  if (best) MB2_CUDA_TRY(cudaMemcpy(best, m->best.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (second) MB2_CUDA_TRY(cudaMemcpy(second, m->second.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (status) MB2_CUDA_TRY(cudaMemcpy(status, m->status.ptr, n, cudaMemcpyDeviceToHost));
  return MIRORR_OK;
}

mirorr_status mirorr_bm_last_diagnostics(mirorr_matcher m, int64_t out[6]) {
  if (!m || !out) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!m->has_results) { set_error("no results: call GetOffsets first"); return MIRORR_ESTATE; }
  unsigned int ctl[8] = {0};
  MB2_CUDA_TRY(cudaSetDevice(m->ctx->device));
  if (is16(m->storage)) {
    unsigned int c16[2] = {0, 0};
    MB2_TRY(match16_counts(m->ctx->bm16, m->ctx->stream, c16));
    out[0] = 0;
    out[1] = 0;
    out[2] = m->kept;
    out[3] = m->last.nblocks;
    out[4] = c16[0];
    out[5] = c16[1];
    return MIRORR_OK;
  }
  MB2_CUDA_TRY(cudaMemcpy(ctl, m->ctx->bmw.ncc_ctl.ptr, sizeof(ctl), cudaMemcpyDeviceToHost));
  out[0] = ctl[2];
  out[1] = ctl[1];
  out[2] = m->kept;
  out[3] = m->last.nblocks;
  out[4] = ctl[3];
  out[5] = ctl[0];
  return MIRORR_OK;
}

mirorr_status mirorr_bm_last_timings(mirorr_matcher m, float ms[4]) {
  if (!m || !ms) { set_error("null argument"); return MIRORR_EINVAL; }
  for (int i = 0; i < 4; ++i) ms[i] = m->timings[i];
  return MIRORR_OK;
}

// ---- resampler -----------------------------------------------------------------
mirorr_status mirorr_resample_map(const mirorr_geometry *out_grid, const mirorr_geometry *in_grid,
                                  const double M[9], const double offset[3], double C[9],
                                  double e[3]) {
  if (!out_grid || !in_grid || !M || !offset || !C || !e) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  ResampleMap m;
  if (!make_map(*out_grid, *in_grid, M, offset, m)) {
    set_error("singular input geometry");
    return MIRORR_EINVAL;
  }
  memcpy(C, m.C, sizeof(m.C));
  memcpy(e, m.e, sizeof(m.e));
  return MIRORR_OK;
}

static mirorr_status resample_common(mirorr_ctx c, const int32_t in_size[3], const float *in_image,
                                     const uint8_t *in_mask, const int32_t out_size[3],
                                     const double C[9], const double e[3], float *out_image,
                                     uint8_t *out_mask, bool nearest) {
  if (!c || !in_size || !out_size || !C || !e) { set_error("null argument"); return MIRORR_EINVAL; }
  if ((in_image && !out_image) || (in_mask && !out_mask)) {
    set_error("output buffer missing");
    return MIRORR_EINVAL;
  }
  for (int d = 0; d < 3; ++d)
    if (in_size[d] <= 0 || out_size[d] <= 0) { set_error("empty volume"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  long long ni = vox(in_size), no = vox(out_size);
  DevBuf di, dm, oi, om;
  mirorr_status st = MIRORR_OK;
  const float *pi = nullptr;
  const uint8_t *pm = nullptr;
  if (in_image) {
    if ((st = upload(c, di, in_image, sizeof(float) * ni)) != MIRORR_OK) goto done;
    pi = di.as<float>();
    if ((st = oi.ensure(sizeof(float) * no)) != MIRORR_OK) goto done;
  }
  if (in_mask) {
    if ((st = upload(c, dm, in_mask, ni)) != MIRORR_OK) goto done;
    pm = dm.as<uint8_t>();
    if ((st = om.ensure(no)) != MIRORR_OK) goto done;
  }
  {
    ResampleMap m;
    memcpy(m.C, C, sizeof(m.C));
    memcpy(m.e, e, sizeof(m.e));
    // image and mask share the input grid and the map: one launch for both
    if ((st = launch_resample(in_size, pi, pm, out_size, m, pi ? oi.as<float>() : nullptr,
                              pm ? om.as<uint8_t>() : nullptr, c->stream, nearest)) != MIRORR_OK)
      goto done;
    if (pi && cudaMemcpyAsync(out_image, oi.ptr, sizeof(float) * no, cudaMemcpyDeviceToHost,
                              c->stream) != cudaSuccess) { st = MIRORR_ECUDA; goto done; }
    if (pm && cudaMemcpyAsync(out_mask, om.ptr, no, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) {
      st = MIRORR_ECUDA;
      goto done;
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
      set_error("resample failed: %s", cudaGetErrorString(cudaGetLastError()));
      st = MIRORR_ECUDA;
    }
  }
done:
  cudaStreamSynchronize(c->stream);
  di.release(); dm.release(); oi.release(); om.release();
  return st;
}

mirorr_status mirorr_resample(mirorr_ctx c, const int32_t in_size[3], const float *in_image,
                              const uint8_t *in_mask, const int32_t out_size[3], const double C[9],
                              const double e[3], float *out_image, uint8_t *out_mask) {
  return resample_common(c, in_size, in_image, in_mask, out_size, C, e, out_image, out_mask, false);
}

mirorr_status mirorr_resample_nearest(mirorr_ctx c, const int32_t in_size[3], const float *in_image,
                                      const uint8_t *in_mask, const int32_t out_size[3],
                                      const double C[9], const double e[3], float *out_image,
                                      uint8_t *out_mask) {
  return resample_common(c, in_size, in_image, in_mask, out_size, C, e, out_image, out_mask, true);
}

// Final resampling with the B-spline (bspline) or windowed-sinc interpolator:
// image only, host buffers in and out.
static mirorr_status resample_final(mirorr_ctx c, const int32_t in_size[3], const float *in_image,
                                    const int32_t out_size[3], const double C[9],
                                    const double e[3], float *out_image, bool bspline) {
  if (!c || !in_size || !out_size || !C || !e || !in_image || !out_image) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  for (int d = 0; d < 3; ++d)
    if (in_size[d] <= 0 || out_size[d] <= 0) { set_error("empty volume"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  const long long ni = vox(in_size), no = vox(out_size);
  DevBuf di, coef, oi;
  auto run = [&]() -> mirorr_status {
    MB2_TRY(upload(c, di, in_image, sizeof(float) * ni));
    MB2_TRY(oi.ensure(sizeof(float) * no));
    ResampleMap m;
    memcpy(m.C, C, sizeof(m.C));
    memcpy(m.e, e, sizeof(m.e));
    if (bspline) {
      MB2_TRY(coef.ensure(sizeof(double) * ni));
      MB2_TRY(launch_resample_bspline(in_size, di.as<float>(), out_size, m, coef.as<double>(),
                                      oi.as<float>(), c->stream));
    } else {
      MB2_TRY(launch_resample_sinc(in_size, di.as<float>(), out_size, m, oi.as<float>(),
                                   c->stream));
    }
    MB2_CUDA_TRY(cudaMemcpyAsync(out_image, oi.ptr, sizeof(float) * no, cudaMemcpyDeviceToHost,
                                 c->stream));
    MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MIRORR_OK;
  };
  const mirorr_status st = run();
  cudaStreamSynchronize(c->stream);  // nothing in flight uses the buffers below
  di.release();
  coef.release();
  oi.release();
  return st;
}

mirorr_status mirorr_resample_device(mirorr_ctx c, const int32_t in_size[3], const float *in_image,
                                     const uint8_t *in_mask, const int32_t out_size[3],
                                     const double C[9], const double e[3], float *out_image,
                                     uint8_t *out_mask, int32_t nearest) {
  if (!c || !in_size || !out_size || !C || !e || (!in_image && !in_mask) ||
      (in_image && !out_image) || (in_mask && !out_mask)) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  for (int d = 0; d < 3; ++d)
    if (in_size[d] <= 0 || out_size[d] <= 0) { set_error("empty volume"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  ResampleMap m;
  memcpy(m.C, C, sizeof(m.C));
  memcpy(m.e, e, sizeof(m.e));
  return launch_resample(in_size, in_image, in_mask, out_size, m, in_image ? out_image : nullptr,
                         in_mask ? out_mask : nullptr, c->stream, nearest != 0);
}

mirorr_status mirorr_resample_bspline(mirorr_ctx c, const int32_t in_size[3],
                                      const float *in_image, const int32_t out_size[3],
                                      const double C[9], const double e[3], float *out_image) {
  return resample_final(c, in_size, in_image, out_size, C, e, out_image, true);
}

mirorr_status mirorr_resample_sinc(mirorr_ctx c, const int32_t in_size[3], const float *in_image,
                                   const int32_t out_size[3], const double C[9],
                                   const double e[3], float *out_image) {
  return resample_final(c, in_size, in_image, out_size, C, e, out_image, false);
}

// ---- LTS ---------------------------------------------------------------------------
static mirorr_status lts_common(mirorr_ctx c, mirorr_transform *t, mirorr_transform *t12f,
                                mirorr_transform *t12b, size_t n, const double *init,
                                const double *moved, double lts_keep, int32_t *inner, bool sym) {
  if (!c || !t || (n && (!init || !moved)) || (sym && (!t12f || !t12b))) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  if (!(lts_keep > 0.0 && lts_keep <= 1.0)) { set_error("lts_keep must lie in (0, 1]"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  LtsState hs;
  memset(&hs, 0, sizeof(hs));
  if (!from_public(*t, hs.tfm)) { set_error("bad transform kind"); return MIRORR_EINVAL; }
  hs.kind = t->kind;
  hs.symmetric = sym ? 1 : 0;
  hs.lts_keep = lts_keep;
  if (sym) {
    if (!from_public(*t12f, hs.t12f) || !from_public(*t12b, hs.t12b)) {
      set_error("bad transform kind");
      return MIRORR_EINVAL;
    }
  }
  MB2_TRY(ensure_pts(c, (long long)n));
  if (n) {
    MB2_CUDA_TRY(cudaMemcpyAsync(c->pts_i.ptr, init, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    MB2_CUDA_TRY(cudaMemcpyAsync(c->pts_m.ptr, moved, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  }
  long long cnt[4] = {(long long)n, 0, 0, 0};
  MB2_CUDA_TRY(cudaMemcpyAsync(c->counts.ptr, cnt, sizeof(cnt), cudaMemcpyHostToDevice, c->stream));
  int it = 0;
  long long used = 0;
  MB2_TRY(lts_run(c->ltsw, hs, c->pts_i.as<double>(), c->pts_m.as<double>(),
                  c->counts.as<long long>(), (long long)n, c->stream, &it, &used));
  if (inner) *inner = it;
  to_public(hs.tfm, *t);
  if (sym) {
    to_public(hs.t12f, *t12f);
    to_public(hs.t12b, *t12b);
  }
  return MIRORR_OK;
}

mirorr_status mirorr_lts_classic(mirorr_ctx c, mirorr_transform *t, size_t n, const double *init,
                                 const double *moved, double lts_keep, int32_t *inner) {
  return lts_common(c, t, nullptr, nullptr, n, init, moved, lts_keep, inner, false);
}

mirorr_status mirorr_lts_symmetric(mirorr_ctx c, mirorr_transform *t, mirorr_transform *t12f,
                                   mirorr_transform *t12b, size_t n, const double *init,
                                   const double *moved, double lts_keep, int32_t *inner) {
  return lts_common(c, t, t12f, t12b, n, init, moved, lts_keep, inner, true);
}

// True when [p, p + bytes) lies inside one device (or managed) allocation
// usable on device dev.  The allocation's extent comes from the driver's
// cuMemGetAddressRange, looked up through the runtime's entry-point query so
// the library needs no link-time dependency on libcuda.
typedef CUresult (*GetAddressRangeFn)(CUdeviceptr *, size_t *, CUdeviceptr);

static bool device_range_on(const void *p, size_t bytes, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type != cudaMemoryTypeManaged && !(at.type == cudaMemoryTypeDevice && at.device == dev))
    return false;
  static GetAddressRangeFn range_fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &fn, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      range_fn = reinterpret_cast<GetAddressRangeFn>(fn);
    cudaGetLastError();
  });
  if (!range_fn) return false;
  CUdeviceptr base = 0;
  size_t size = 0;
  if (range_fn(&base, &size, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) return false;
  const uintptr_t lo = (uintptr_t)p, end = (uintptr_t)base + size;
  return lo >= (uintptr_t)base && bytes <= end - lo;
}

mirorr_status mirorr_lts_noalloc(mirorr_ctx c, mirorr_transform *t, mirorr_transform *t12f,
                                 mirorr_transform *t12b, size_t n, const double *init,
                                 const double *moved, double lts_keep, int32_t *inner) {
  if (!c || !t || (n && (!init || !moved)) || ((t12f == nullptr) != (t12b == nullptr))) {
    set_error("null argument (t12f and t12b must both be given or both be NULL)");
    return MIRORR_EINVAL;
  }
  const bool sym = t12f != nullptr;
  if (!(lts_keep > 0.0 && lts_keep <= 1.0)) { set_error("lts_keep must lie in (0, 1]"); return MIRORR_EINVAL; }
  if (n > (size_t)MIRORR_LTS_NOALLOC_MAX_POINTS) {
    set_error("%zu point pairs exceed the no-allocation LTS limit of %d", n,
              (int)MIRORR_LTS_NOALLOC_MAX_POINTS);
    return MIRORR_ERANGE;
  }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  if (n) {
    if (((uintptr_t)init | (uintptr_t)moved) & 7u) {
      set_error("point arrays must be 8-byte aligned");
      return MIRORR_EINVAL;
    }
    if (!device_range_on(init, sizeof(double) * 3 * n, c->device) ||
        !device_range_on(moved, sizeof(double) * 3 * n, c->device)) {
      set_error("point arrays must be device memory on the context's device %d, each holding "
                "at least n x 3 doubles", c->device);
      return MIRORR_EINVAL;
    }
  }
  LtsState hs;
  memset(&hs, 0, sizeof(hs));
  if (!from_public(*t, hs.tfm)) { set_error("bad transform kind"); return MIRORR_EINVAL; }
  hs.kind = t->kind;
  hs.symmetric = sym ? 1 : 0;
  hs.lts_keep = lts_keep;
  if (sym) {
    if (!from_public(*t12f, hs.t12f) || !from_public(*t12b, hs.t12b)) {
      set_error("bad transform kind");
      return MIRORR_EINVAL;
    }
  }
  int it = 0;
  MB2_TRY(lts_run_noalloc(hs, init, moved, (long long)n, c->stream, &it));
  if (inner) *inner = it;
  to_public(hs.tfm, *t);
  if (sym) {
    to_public(hs.t12f, *t12f);
    to_public(hs.t12b, *t12b);
  }
  return MIRORR_OK;
}

// ---- registration ----------------------------------------------------------------
mirorr_status mirorr_reg_default_params(mirorr_reg_params *p) {
  if (!p) { set_error("null argument"); return MIRORR_EINVAL; }
  memset(p, 0, sizeof(*p));
  p->symmetric = 1;
  p->kind = KIND_RIGID;
  p->levels = 0;
  p->iterations = 5;
  p->min_length = 32;
  mirorr_bm_default_params(&p->bm);
  p->bm.nhood_gap = 3;
  p->bm.nhood_width = 7;
  p->lts_keep = 0.5;
  return MIRORR_OK;
}

mirorr_status mirorr_register_device(mirorr_ctx c, const mirorr_geometry *fg, const void *fixed,
                                     const uint8_t *fmask, const mirorr_geometry *mg,
                                     const void *moving, const uint8_t *mmask,
                                     const mirorr_reg_params *p, const mirorr_transform *init,
                                     mirorr_transform *result, mirorr_reg_stats *stats) {
  if (!c) { set_error("null argument"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  return register_impl(c, fg, fixed, fmask, mg, moving, mmask, p, init, result, stats);
}

mirorr_status mirorr_register(mirorr_ctx c, const mirorr_geometry *fg, const void *fixed,
                              const uint8_t *fmask, const mirorr_geometry *mg, const void *moving,
                              const uint8_t *mmask, const mirorr_reg_params *p,
                              const mirorr_transform *init, mirorr_transform *result,
                              mirorr_reg_stats *stats) {
  if (!c || !fg || !mg || !fixed || !moving || !p) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!valid_geom(fg) || !valid_geom(mg)) { set_error("invalid image geometry"); return MIRORR_EINVAL; }
  if (p->storage != MIRORR_DTYPE_F32 && !is16(p->storage)) {
    set_error("storage must be MIRORR_DTYPE_F32, _BF16 or _F16 (got %d)", p->storage);
    return MIRORR_EINVAL;
  }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  auto t0 = std::chrono::steady_clock::now();
  const size_t es = elem_size(p->storage);
  MB2_TRY(upload(c, c->up_f, fixed, es * vox(fg->size)));
  MB2_TRY(upload(c, c->up_m, moving, es * vox(mg->size)));
  const uint8_t *dfm = nullptr, *dmm = nullptr;
  if (fmask) { MB2_TRY(upload(c, c->up_fm, fmask, vox(fg->size))); dfm = c->up_fm.as<uint8_t>(); }
  if (mmask) { MB2_TRY(upload(c, c->up_mm, mmask, vox(mg->size))); dmm = c->up_mm.as<uint8_t>(); }
  mirorr_status s = register_impl(c, fg, c->up_f.ptr, dfm, mg, c->up_m.ptr, dmm, p, init, result,
                                  stats);
  if (s == MIRORR_OK && stats) {
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    stats->h2d_bytes += (int64_t)(es * (vox(fg->size) + vox(mg->size)) +
                                  (fmask ? vox(fg->size) : 0) + (mmask ? vox(mg->size) : 0));
  }
  return s;
}

mirorr_status mirorr_pyramid_schedule(const mirorr_geometry *fg, const mirorr_geometry *mg,
                                      int32_t min_length, int32_t max_levels, int32_t *n_levels,
                                      int32_t moving_factors[16][3], int32_t fixed_factors[16][3]) {
  if (!fg || !mg || !n_levels || !moving_factors || !fixed_factors) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  if (!valid_geom(fg) || !valid_geom(mg)) { set_error("invalid geometry"); return MIRORR_EINVAL; }
  int sm[16][3], sf[16][3];
  int n = pyramid_schedule(*fg, *mg, min_length > 0 ? min_length : 32, max_levels, sm, sf);
  *n_levels = n;
  for (int l = 0; l < n; ++l)
    for (int d = 0; d < 3; ++d) { moving_factors[l][d] = sm[l][d]; fixed_factors[l][d] = sf[l][d]; }
  return MIRORR_OK;
}

mirorr_status mirorr_pyramid_level(mirorr_ctx c, const mirorr_geometry *ig, const float *in,
                                   const int32_t factors[3], mirorr_geometry *og, float *out,
                                   size_t out_capacity) {
  if (!c || !ig || !in || !factors || !og || !out) { set_error("null argument"); return MIRORR_EINVAL; }
  if (!valid_geom(ig)) { set_error("invalid geometry"); return MIRORR_EINVAL; }
  for (int d = 0; d < 3; ++d)
    if (factors[d] < 1) { set_error("factors must be >= 1"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  mirorr_geometry g;
  level_geometry(*ig, factors, g);
  if ((size_t)vox(g.size) > out_capacity) {
    *og = g;
    set_error("output capacity too small");
    return MIRORR_ERANGE;
  }
  MB2_TRY(upload(c, c->up_f, in, sizeof(float) * vox(ig->size)));
  const void *lp = nullptr;
  int lt = MIRORR_DTYPE_F32;
  MB2_TRY(make_level(c, *ig, c->up_f.ptr, MIRORR_DTYPE_F32, factors, g, c->lvl_f, &lp, &lt));
  MB2_CUDA_TRY(cudaMemcpyAsync(out, lp, sizeof(float) * vox(g.size), cudaMemcpyDeviceToHost, c->stream));
  MB2_CUDA_TRY(cudaStreamSynchronize(c->stream));
  *og = g;
  return MIRORR_OK;
}

}  // extern "C"

// ---- batched and served registrations ---------------------------------------
//
// A mirorr_batch holds up to max_slots registration requests on the device at
// once, each with its inputs, pyramid level, middle-space images, matcher
// buffers, point pairs and fit state.  A round advances every running
// request by one block-matching iteration with one launch per stage for all
// of them: the resampling passes, the 16-bit search of every matcher call
// (box statistics, window-AND, base blocks, the tensor-core search over all
// calls' tiles in one persistent launch, the direct search), the
// post-filters and the LTS fits (one cooperative launch, a group of CTAs
// per request).  The host reads the fit states back once per round and
// advances each request's iteration, level and convergence as the
// registration methods do (itkMirorrRegistrationMethod.txx:598-658,
// itkSymMirorrRegistrationMethod.txx:458-720, itkMirorrPyramidImplement.txx:
// 107-145).  When the set of requests and their levels is unchanged from the
// round before, the round's launch sequence is replayed from a CUDA graph
// captured once (the per-round index maps and fit states come through
// pinned host buffers the graph's copies read).
namespace {

constexpr int kLtsCtas = 2;  // CTAs per LTS fit in the batched launch

struct BatchCallBufs {
  DevBuf stats, wand, prep, xs, chunked, fb, best, second, match, status, tiles;
  BmWork sel;  // variance selection (var, selected, select_state, hist) when keep < 1
};

struct BatchSlot {
  int state = 0;  // 0 free, 1 running, 2 finished, 3 failed
  int64_t id = -1;
  mirorr_status fail = MIRORR_OK;
  std::string fail_msg;
  mirorr_reg_params p{};
  mirorr_geometry fg{}, mg{};
  DevBuf in_f, in_m, in_fm, in_mm;
  bool has_fm = false, has_mm = false;
  int nl = 0, lev = 0, it = 0;
  int sf[16][3], sm[16][3];
  double params[12];
  Tfm tfm, t12f, t12b, fixed_tr, moving_tr;
  double initial_center[3];
  double last[12];
  bool level_ready = false;
  mirorr_geometry lf{}, lm{}, grid_f{}, grid_m{};
  DevBuf lvl_f, lvl_m;
  BmGeom g{};
  DevBuf img_b, img_s, msk_b, msk_s;
  BatchCallBufs call[2];
  DevBuf pts_i, pts_m, lts_scratch;
  long long cap_blocks = 0;  // blocks the buffers hold (the finest level's)
  mirorr_reg_stats stats{};
  std::chrono::steady_clock::time_point t0;
  size_t bytes = 0;
  // one device allocation holds every buffer above (they are views into it)
  void *arena = nullptr;
  size_t arena_bytes = 0;
};

size_t slot_bytes(const mirorr_geometry &fg, const mirorr_geometry &mg, const mirorr_reg_params &p,
                  bool fm, bool mm, long long max_vox, long long max_blocks) {
  const size_t es = elem_size(p.storage);
  const size_t nf = (size_t)vox(fg.size), nm = (size_t)vox(mg.size);
  const size_t ncall = p.symmetric ? 2 : 1;
  const size_t V = (size_t)max_vox, NB = (size_t)max_blocks;
  size_t b = es * (nf + nm) + (fm ? nf : 0) + (mm ? nm : 0);  // inputs
  b += 4 * (nf + nm);                                          // float32 levels
  b += 2 * es * V + 2 * V;                                     // middle-space images, masks
  // statistics with even-pitch rows (<= 8 V (1 + 1 / nx), nx >= 4), window-AND,
  // x-chunked copy, per-block records
  b += ncall * (10 * V + 3 * V / 2 + (32 + 256 + 4 + 13) * NB + 2 * V + 64 * 1024);
  if (p.bm.block_keep < 1.0) b += ncall * (17 * NB + 2048);  // variance selection
  b += 2 * 3 * 8 * ncall * NB;                                 // point pairs
  b += lts_fit_scratch_bytes((long long)(ncall * NB), kLtsCtas);
  return b;
}

}  // namespace

struct mirorr_batch_s {
  mirorr_ctx c = nullptr;
  int max_slots = 0;
  size_t budget = 0, used = 0;
  std::vector<BatchSlot> slots;
  int64_t next_id = 1;
  bool params_set = false;
  mirorr_bm_params bm{};
  int storage = MIRORR_DTYPE_BF16;
  // per-round staging (pinned) and device copies
  HostBuf h_jobs, h_calls, h_pf, h_states, h_rd;
  DevBuf d_jobs, d_pf, d_states, d_counts, d_ctl, d_calls, d_lts_args;
  HostBuf h_lts_args;
  std::vector<LtsFit> fits;
  std::vector<int> fit_slot, call_slot;
  // graph of the last round's launch sequence
  bool graphs = true;
  cudaGraphExec_t gexec = nullptr;
  std::vector<long long> gkey;
  int64_t rounds = 0, replays = 0, captures = 0, updates = 0;
  // arenas of finished requests, kept for the next ones (by size); their
  // bytes plus the live requests' stay within the budget
  std::multimap<size_t, void *> pool;
  size_t pool_bytes = 0;
  // host-clock seconds: level setup, descriptors and graph work, launch to
  // synchronisation, advancing the requests
  double t_setup = 0, t_issue = 0, t_device = 0, t_advance = 0;
};

namespace {

// Sets up slot s's current level: the level images (float32), the middle
// space, the block grid and, for the symmetric method, the half-space
// transforms (symmetric_level's preamble).
mirorr_status batch_setup_level(mirorr_batch b, BatchSlot &s) {
  mirorr_ctx c = b->c;
  cudaStream_t st = c->stream;
  const void *pf = nullptr, *pm = nullptr;
  int tf = 0, tm = 0;
  MB2_TRY(make_level(c, s.fg, s.in_f.ptr, s.p.storage, s.sf[s.lev], s.lf, s.lvl_f, &pf, &tf));
  if (tf != MIRORR_DTYPE_F32) {
    MB2_TRY(s.lvl_f.ensure(sizeof(float) * vox(s.lf.size)));
    MB2_TRY(launch_from16(pf, s.lvl_f.as<float>(), vox(s.lf.size), tf, st));
  }
  MB2_TRY(make_level(c, s.mg, s.in_m.ptr, s.p.storage, s.sm[s.lev], s.lm, s.lvl_m, &pm, &tm));
  if (tm != MIRORR_DTYPE_F32) {
    MB2_TRY(s.lvl_m.ensure(sizeof(float) * vox(s.lm.size)));
    MB2_TRY(launch_from16(pm, s.lvl_m.as<float>(), vox(s.lm.size), tm, st));
  }
  double cf[3], cm[3], origin[3], spacing[3];
  int size[3];
  center_of(s.lf, cf);
  center_of(s.lm, cm);
  for (int d = 0; d < 3; ++d) {
    origin[d] = s.p.symmetric ? ((s.lf.origin[d] - cf[d]) + (s.lm.origin[d] - cm[d])) / 2.0
                              : cm[d] + ((s.lf.origin[d] - cf[d]) + (s.lm.origin[d] - cm[d])) / 2.0;
    spacing[d] = (s.lf.spacing[d] + s.lm.spacing[d]) / 2.0;
    size[d] = (int)(((double)s.lf.size[d] + (double)s.lm.size[d] + 0.5) / 2.0);
  }
  grid_geom(origin, spacing, size, s.lf.direction, s.grid_f);
  grid_geom(origin, spacing, size, s.lm.direction, s.grid_m);
  if (!bm_geometry(size, (int)s.p.bm.block_width, (int)s.p.bm.block_gap, (int)s.p.bm.nhood_gap,
                   (int)s.p.bm.nhood_width, s.g)) {
    set_error("middle-space image smaller than one block");
    return MIRORR_EINVAL;
  }
  tfm_set_params(s.tfm, s.params);
  if (s.p.symmetric) {
    for (int d = 0; d < 3; ++d) s.initial_center[d] = s.tfm.c[d];
    tfm_center_to_origin(s.tfm);
    tfm_identity(s.fixed_tr, KIND_RIGID);
    tfm_identity(s.moving_tr, KIND_RIGID);
    double pfx[6] = {0, 0, 0, cf[0], cf[1], cf[2]}, pmv[6] = {0, 0, 0, cm[0], cm[1], cm[2]};
    tfm_set_params(s.fixed_tr, pfx);
    tfm_set_params(s.moving_tr, pmv);
    Tfm ifixed;
    tfm_inverse(s.fixed_tr, ifixed);
    tfm_compose(s.tfm, ifixed, false);
    tfm_compose(s.tfm, s.moving_tr, true);
    half_space(s.tfm, s.t12f, s.t12b);
  }
  tfm_params(s.tfm, s.last);
  s.it = 0;
  s.level_ready = true;
  return MIRORR_OK;
}

void batch_centered(const BatchSlot &s, Tfm &cF, Tfm &cB) {
  double prm[12];
  tfm_identity(cF, s.tfm.kind);
  tfm_identity(cB, s.tfm.kind);
  tfm_params(s.t12f, prm);
  tfm_set_params(cF, prm);
  tfm_compose(cF, s.fixed_tr, false);
  tfm_params(s.t12b, prm);
  tfm_set_params(cB, prm);
  tfm_compose(cB, s.moving_tr, false);
}

// End of slot s's level: the symmetric method composes the full transform
// back (symmetric_level's epilogue); the parameters carry to the next level.
void batch_end_level(BatchSlot &s) {
  if (s.p.symmetric) {
    Tfm cF, cB, ib;
    batch_centered(s, cF, cB);
    tfm_inverse(cB, ib);
    tfm_identity(s.tfm, s.tfm.kind);
    tfm_compose(s.tfm, ib, true);
    tfm_compose(s.tfm, cF, false);
    tfm_update_center(s.tfm, s.initial_center);
  }
  if (s.lev < 16) s.stats.iterations_run[s.lev] = s.it;
  tfm_params(s.tfm, s.params);
  s.level_ready = false;
  ++s.lev;
  if (s.lev >= s.nl) {
    tfm_set_params(s.tfm, s.params);
    s.stats.levels_run = s.nl;
    s.stats.seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - s.t0).count();
    s.state = 2;
  }
}

void batch_fail(mirorr_batch b, BatchSlot &s, mirorr_status st, const char *msg) {
  s.state = 3;
  s.fail = st;
  s.fail_msg = msg;
  (void)b;
}

// Frees cached arenas, largest first, while the live requests and the cache
// together exceed the budget.
void pool_trim(mirorr_batch b, size_t extra) {
  while (!b->pool.empty() && b->used + b->pool_bytes + extra > b->budget) {
    auto last = std::prev(b->pool.end());
    cudaFree(last->second);
    b->pool_bytes -= last->first;
    b->pool.erase(last);
  }
}

// The slot's buffers (each of `list`'s sizes, 256-byte aligned) as views into
// one arena: the smallest cached arena that holds them, else a new one.
mirorr_status slot_carve(mirorr_batch b, BatchSlot &s,
                         const std::vector<std::pair<DevBuf *, size_t>> &list) {
  auto up = [](size_t v) { return (std::max<size_t>(v, 1) + 255) / 256 * 256; };
  size_t total = 0;
  for (auto &e : list) total += up(e.second);
  void *p = nullptr;
  size_t pb = 0;
  auto it = b->pool.lower_bound(total);
  if (it != b->pool.end()) {
    p = it->second;
    pb = it->first;
    b->pool_bytes -= pb;
    b->pool.erase(it);
  } else {
    pool_trim(b, 0);
    cudaError_t e = cudaMalloc(&p, total);
    if (e != cudaSuccess) {
      cudaGetLastError();
      pool_trim(b, b->budget);  // everything cached
      e = cudaMalloc(&p, total);
      if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc(%zu) for a batch request failed: %s", total, cudaGetErrorString(e));
        return MIRORR_ENOMEM;
      }
    }
    pb = total;
  }
  s.arena = p;
  s.arena_bytes = pb;
  size_t off = 0;
  for (auto &e : list) {
    e.first->ptr = static_cast<char *>(p) + off;
    e.first->bytes = up(e.second);
    off += up(e.second);
  }
  return MIRORR_OK;
}

// The slot's arena goes back to the cache; its buffers were views into it.
void batch_release(mirorr_batch b, BatchSlot &s) {
  if (s.arena) {
    b->pool.insert({s.arena_bytes, s.arena});
    b->pool_bytes += s.arena_bytes;
  }
  b->used -= s.bytes;
  s = BatchSlot();
  pool_trim(b, 0);
}

// Host-side check, before any launch, that every buffer a round's
// descriptors address is large enough for the extent the kernels will touch.
mirorr_status batch_check_slot(mirorr_ctx c, const BatchSlot &s) {
  const long long nvox = vox(s.grid_f.size), nb = s.g.nblocks;
  const size_t es = elem_size(s.p.storage);
  const int ncall = s.p.symmetric ? 2 : 1;
  auto need = [&](const DevBuf &x, size_t n, const char *what) -> bool {
    if (x.bytes >= n && x.ptr) return true;
    set_error("internal: slot buffer %s holds %zu bytes, the round needs %zu", what, x.bytes, n);
    return false;
  };
  bool ok = need(s.img_b, es * nvox, "img_b") && need(s.img_s, es * nvox, "img_s") &&
            need(s.msk_b, nvox, "msk_b") && need(s.msk_s, nvox, "msk_s") &&
            need(s.lvl_f, sizeof(float) * vox(s.lf.size), "lvl_f") &&
            need(s.lvl_m, sizeof(float) * vox(s.lm.size), "lvl_m") &&
            need(s.pts_i, sizeof(double) * 3 * ncall * nb, "pts_i") &&
            need(s.pts_m, sizeof(double) * 3 * ncall * nb, "pts_m") &&
            need(s.lts_scratch, lts_fit_scratch_bytes(ncall * nb, kLtsCtas), "lts_scratch");
  if (ok && !s.has_fm) ok = need(c->ones, vox(s.fg.size), "ones (fixed)");
  if (ok && !s.has_mm) ok = need(c->ones, vox(s.mg.size), "ones (moving)");
  for (int k = 0; ok && k < ncall; ++k) {
    Match16Call mc;
    memset(&mc, 0, sizeof(mc));
    prepare16(s.g, mc);
    const BatchCallBufs &cb = s.call[k];
    ok = need(cb.stats, match16_stats_bytes(mc), "stats") &&
         need(cb.wand, match16_wand_bytes(mc), "wand") &&
         need(cb.prep, sizeof(Prep16) * nb, "prep") && need(cb.xs, 256 * (size_t)nb, "xs") &&
         need(cb.fb, sizeof(int) * nb, "fb") && need(cb.best, sizeof(float) * nb, "best") &&
         need(cb.second, sizeof(float) * nb, "second") &&
         need(cb.match, sizeof(int32_t) * nb, "match") && need(cb.status, nb, "status") &&
         need(cb.tiles, sizeof(unsigned int) * ((nb + 2047) / 2048 + 1), "tiles") &&
         (!mc.tensor || need(cb.chunked, match16_chunk_bytes(mc), "chunked")) &&
         (!(s.p.bm.block_keep < 1.0) ||
          (need(cb.sel.var, selection_var_bytes(nb), "selection keys") &&
           need(cb.sel.selected, (size_t)nb, "selection flags") &&
           need(cb.sel.select_state, selection_state_bytes(), "selection state")));
  }
  return ok ? MIRORR_OK : MIRORR_EINVAL;
}

// The round's launch sequence (also what a graph captures).
mirorr_status batch_issue(mirorr_batch b, int njobs, long long max_vox, int ncalls, int nfits,
                          long long max_blocks) {
  mirorr_ctx c = b->c;
  cudaStream_t st = c->stream;
  const int S = b->max_slots;
  MB2_CUDA_TRY(cudaMemcpyAsync(b->d_jobs.ptr, b->h_jobs.ptr, sizeof(ResampleJob) * njobs,
                               cudaMemcpyHostToDevice, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(b->d_pf.ptr, b->h_pf.ptr, sizeof(PfCall) * ncalls,
                               cudaMemcpyHostToDevice, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(b->d_states.ptr, b->h_states.ptr, sizeof(LtsState) * S,
                               cudaMemcpyHostToDevice, st));
  MB2_CUDA_TRY(cudaMemsetAsync(b->d_counts.ptr, 0, sizeof(long long) * 4 * S, st));
  MB2_CUDA_TRY(cudaMemsetAsync(b->d_ctl.ptr, 0, sizeof(unsigned int) * 4 * 2 * S, st));
  MB2_TRY(launch_resample_batch(b->d_jobs.as<ResampleJob>(), njobs, max_vox, st));
  // the variance selection of the calls of requests that keep a fraction of
  // their blocks (on this iteration's resampled base images)
  {
    const Match16Call *calls = b->h_calls.as<Match16Call>();
    int prev = -1;
    for (int ci = 0; ci < ncalls; ++ci) {
      const int si = b->call_slot[ci];
      const int k = si == prev ? 1 : 0;
      prev = si;
      BatchSlot &s = b->slots[si];
      if (!(s.p.bm.block_keep < 1.0)) continue;
      const uint8_t *sel = nullptr;
      MB2_TRY(launch_variance_selection(s.g, calls[ci].base, s.p.bm.block_keep, s.call[k].sel, &sel, st,
                                        b->storage, calls[ci].ctl + 2, c->ltsw.spin_limit));
    }
  }
  MB2_TRY(launch_match16_batch(b->storage, ncalls, b->h_calls.as<Match16Call>(), b->d_calls, st,
                               true));
  MB2_TRY(launch_postfilter_batch(b->d_pf.as<PfCall>(), ncalls, max_blocks, st));
  MB2_TRY(lts_batch_launch(b->fits.data(), nfits, kLtsCtas, c->ltsw.spin_limit, b->d_lts_args,
                           b->h_lts_args, st));
  // read back: fit states, point counts, the search's and the fits' give-up flags
  unsigned char *rd = b->h_rd.as<unsigned char>();
  MB2_CUDA_TRY(cudaMemcpyAsync(rd, b->d_states.ptr, sizeof(LtsState) * S, cudaMemcpyDeviceToHost, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(rd + sizeof(LtsState) * S, b->d_counts.ptr, sizeof(long long) * 4 * S,
                               cudaMemcpyDeviceToHost, st));
  MB2_CUDA_TRY(cudaMemcpyAsync(rd + sizeof(LtsState) * S + sizeof(long long) * 4 * S, b->d_ctl.ptr,
                               sizeof(unsigned int) * 4 * 2 * S, cudaMemcpyDeviceToHost, st));
  return MIRORR_OK;
}

// One round over every running request.
mirorr_status batch_round(mirorr_batch b, int *running, int *finished) {
  mirorr_ctx c = b->c;
  cudaStream_t st = c->stream;
  const int S = b->max_slots;
  int nrun = 0;
  long long max_in = 0;
  for (auto &s : b->slots)
    if (s.state == 1) {
      ++nrun;
      max_in = std::max(max_in, (long long)std::max(vox(s.fg.size), vox(s.mg.size)));
    }
  if (running) *running = nrun;
  if (finished) *finished = 0;
  if (!nrun) return MIRORR_OK;
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point z) {
    return std::chrono::duration<double>(z - a).count();
  };
  const clk::time_point t0 = clk::now();
  MB2_TRY(ensure_ones(c, max_in));
  // levels entered this round
  for (auto &s : b->slots) {
    if (s.state != 1 || s.level_ready) continue;
    mirorr_status r = batch_setup_level(b, s);
    if (r != MIRORR_OK) batch_fail(b, s, r, mirorr_last_error());
  }
  const clk::time_point t1 = clk::now();
  b->t_setup += secs(t0, t1);
  ResampleJob *jobs = b->h_jobs.as<ResampleJob>();
  Match16Call *calls = b->h_calls.as<Match16Call>();
  PfCall *pf = b->h_pf.as<PfCall>();
  LtsState *states = b->h_states.as<LtsState>();
  memset(states, 0, sizeof(LtsState) * S);
  b->fits.clear();
  b->fit_slot.clear();
  b->call_slot.clear();
  int nj = 0, nc = 0;
  long long max_vox = 0, max_blocks = 0;
  std::vector<long long> key;
  for (int si = 0; si < S; ++si) {
    BatchSlot &s = b->slots[si];
    if (s.state != 1) continue;
    // a slot reused by a later request has other buffers: the request id
    // (not the slot) keys the graph
    key.push_back(s.id);
    key.push_back(s.lev);
    const long long V = vox(s.grid_f.size);
    max_vox = std::max(max_vox, V);
    max_blocks = std::max(max_blocks, s.g.nblocks);
    // ---- resampling passes of this iteration ------------------------------
    Tfm tb, tf;
    if (s.p.symmetric) {
      batch_centered(s, tf, tb);
    } else {
      tfm_identity(tb, KIND_AFFINE);
      tf = s.tfm;
    }
    const uint8_t *fmask = s.has_fm ? s.in_fm.as<uint8_t>() : c->ones.as<uint8_t>();
    const uint8_t *mmask = s.has_mm ? s.in_mm.as<uint8_t>() : c->ones.as<uint8_t>();
    struct Src { const float *img; const mirorr_geometry *lg; const uint8_t *mask;
                 const mirorr_geometry *mgeo; const mirorr_geometry *grid; const Tfm *t;
                 DevBuf *out; DevBuf *outm; };
    Src src[2] = {{s.lvl_m.as<float>(), &s.lm, mmask, &s.mg, &s.grid_m, &tb, &s.img_b, &s.msk_b},
                  {s.lvl_f.as<float>(), &s.lf, fmask, &s.fg, &s.grid_f, &tf, &s.img_s, &s.msk_s}};
    for (auto &q : src) {
      ResampleMap mi, mmp;
      if (!make_map(*q.grid, *q.lg, q.t->M, q.t->off, mi) ||
          !make_map(*q.grid, *q.mgeo, q.t->M, q.t->off, mmp)) {
        batch_fail(b, s, MIRORR_EINVAL, "singular image geometry");
        break;
      }
      ResampleJob &ji = jobs[nj++];
      memset(&ji, 0, sizeof(ji));
      ji.in = q.img;
      ji.out = q.out->ptr;
      for (int d = 0; d < 3; ++d) { ji.in_size[d] = q.lg->size[d]; ji.out_size[d] = q.grid->size[d]; }
      memcpy(ji.C, mi.C, sizeof(mi.C));
      memcpy(ji.e, mi.e, sizeof(mi.e));
      ji.out_dtype = s.p.storage;
      ji.active = 1;
      ResampleJob &jm = jobs[nj++];
      memset(&jm, 0, sizeof(jm));
      jm.inm = q.mask;
      jm.outm = q.outm->as<uint8_t>();
      jm.mask_ones = q.mask == c->ones.as<uint8_t>() ? 1 : 0;
      for (int d = 0; d < 3; ++d) { jm.in_size[d] = q.mgeo->size[d]; jm.out_size[d] = q.grid->size[d]; }
      memcpy(jm.C, mmp.C, sizeof(mmp.C));
      memcpy(jm.e, mmp.e, sizeof(mmp.e));
      jm.active = 1;
    }
    if (s.state != 1) continue;
    // ---- matcher calls: forward, and the swapped one of the symmetric method
    const int ncall = s.p.symmetric ? 2 : 1;
    for (int k = 0; k < ncall; ++k) {
      Match16Call &mc = calls[nc];
      memset(&mc, 0, sizeof(mc));
      prepare16(s.g, mc);
      BatchCallBufs &cb = s.call[k];
      mc.base = k ? s.img_s.ptr : s.img_b.ptr;
      mc.bmask = k ? s.msk_s.as<uint8_t>() : s.msk_b.as<uint8_t>();
      mc.search = k ? s.img_b.ptr : s.img_s.ptr;
      mc.smask = k ? s.msk_b.as<uint8_t>() : s.msk_s.as<uint8_t>();
      mc.selected = s.p.bm.block_keep < 1.0 ? cb.sel.selected.as<uint8_t>() : nullptr;
      mc.stats = cb.stats.as<float2>();
      mc.wand = cb.wand.as<uint8_t>();
      mc.prep = cb.prep.as<Prep16>();
      mc.xs = cb.xs.as<uint32_t>();
      mc.chunked = cb.chunked.as<uint4>();
      mc.best = cb.best.as<float>();
      mc.second = cb.second.as<float>();
      mc.match = cb.match.as<int32_t>();
      mc.status = cb.status.as<uint8_t>();
      mc.ncc_count = reinterpret_cast<unsigned long long *>(b->d_counts.as<long long>() + 4 * si + 2);
      mc.ctl = b->d_ctl.as<unsigned int>() + 4 * (2 * si + k);
      mc.fb_list = cb.fb.as<int>();
      mc.active = 1;
      PfCall &pc = pf[nc];
      memset(&pc, 0, sizeof(pc));
      pc.out = BmOut{mc.best, mc.second, mc.match, mc.status};
      pc.g = s.g;
      const mirorr_geometry &pg_geom = k ? s.grid_f : s.grid_m;
      point_geom(pg_geom.origin, pg_geom.spacing, pg_geom.direction, (int)s.p.bm.block_width, pc.pg);
      // the swapped call's lists go in with roles reversed, after the forward ones
      pc.pts_b = k ? s.pts_m.as<double>() : s.pts_i.as<double>();
      pc.pts_m = k ? s.pts_i.as<double>() : s.pts_m.as<double>();
      pc.tiles = cb.tiles.as<unsigned int>();
      pc.count = b->d_counts.as<long long>() + 4 * si + k;
      pc.offset = k ? b->d_counts.as<long long>() + 4 * si : nullptr;
      pc.active = 1;
      b->call_slot.push_back(si);
      ++nc;
    }
    key.push_back(s.g.nblocks);
    // ---- the fit --------------------------------------------------------------
    LtsState &hs = states[si];
    hs.kind = s.tfm.kind;
    hs.symmetric = s.p.symmetric;
    hs.lts_keep = s.p.lts_keep;
    hs.tfm = s.tfm;
    if (s.p.symmetric) {
      hs.t12f = s.t12f;
      hs.t12b = s.t12b;
    }
    lts_begin(hs);
    LtsFit f;
    f.state = b->d_states.as<LtsState>() + si;
    f.init = s.pts_i.as<double>();
    f.moved = s.pts_m.as<double>();
    f.n_dev = b->d_counts.as<long long>() + 4 * si;
    f.scratch = s.lts_scratch.ptr;
    b->fits.push_back(f);
    b->fit_slot.push_back(si);
  }
  if (nc == 0) return MIRORR_OK;
  for (int si = 0; si < S; ++si)
    if (b->slots[si].state == 1) MB2_TRY(batch_check_slot(c, b->slots[si]));
  // the tile numbering and copy descriptors the tensor launch reads from the
  // call descriptors (a replay copies them from h_calls as written here)
  match16_number_tiles(calls, nc);
  MB2_TRY(match16_prepare_copies(b->storage, calls, nc));
  // ---- launches ---------------------------------------------------------------
  // Replayed from the graph when the set of requests and levels is unchanged.
  // Otherwise the round is captured again; as every round launches the same
  // sequence of nodes (only sizes, grids and arguments differ), the existing
  // executable graph is updated in place, and instantiated anew only when the
  // update is refused.
  const bool same = b->graphs && b->gexec && key == b->gkey;
  if (same) {
    const clk::time_point t2 = clk::now();
    b->t_issue += secs(t1, t2);
    MB2_CUDA_TRY(cudaGraphLaunch(b->gexec, st));
    ++b->replays;
  } else if (b->graphs) {
    MB2_TRY(b->d_calls.ensure(sizeof(Match16Call) * nc));
    MB2_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    mirorr_status r = batch_issue(b, nj, max_vox, nc, (int)b->fits.size(), max_blocks);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (r != MIRORR_OK) {
      if (graph) cudaGraphDestroy(graph);
      return r;
    }
    if (e != cudaSuccess) {
      set_error("capturing the batch round failed: %s", cudaGetErrorString(e));
      return MIRORR_ECUDA;
    }
    bool updated = false;
    if (b->gexec) {
      cudaGraphExecUpdateResultInfo ui;
      if (cudaGraphExecUpdate(b->gexec, graph, &ui) == cudaSuccess) {
        updated = true;
        ++b->updates;
      } else {
        cudaGetLastError();
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
      }
    }
    if (!updated) {
      e = cudaGraphInstantiate(&b->gexec, graph, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        b->gexec = nullptr;
        set_error("instantiating the batch round failed: %s", cudaGetErrorString(e));
        return MIRORR_ECUDA;
      }
      ++b->captures;
    }
    cudaGraphDestroy(graph);
    b->gkey = key;
    const clk::time_point t2 = clk::now();
    b->t_issue += secs(t1, t2);
    MB2_CUDA_TRY(cudaGraphLaunch(b->gexec, st));
  } else {
    const clk::time_point t2 = clk::now();
    b->t_issue += secs(t1, t2);
    MB2_TRY(batch_issue(b, nj, max_vox, nc, (int)b->fits.size(), max_blocks));
  }
  const clk::time_point t3 = clk::now();
  MB2_CUDA_TRY(cudaStreamSynchronize(st));
  const clk::time_point t4 = clk::now();
  b->t_device += secs(t3, t4);
  ++b->rounds;
  // ---- advance every request ----------------------------------------------
  const unsigned char *rd = b->h_rd.as<unsigned char>();
  const LtsState *rs = reinterpret_cast<const LtsState *>(rd);
  const long long *rc = reinterpret_cast<const long long *>(rd + sizeof(LtsState) * S);
  const unsigned int *rctl =
      reinterpret_cast<const unsigned int *>(rd + sizeof(LtsState) * S + sizeof(long long) * 4 * S);
  int nfin = 0;
  for (size_t fi = 0; fi < b->fit_slot.size(); ++fi) {
    const int si = b->fit_slot[fi];
    BatchSlot &s = b->slots[si];
    if (rctl[4 * (2 * si) + 2] || rctl[4 * (2 * si + 1) + 2]) {
      batch_fail(b, s, MIRORR_ETIMEOUT, "a bounded wait of the block search (a tensor copy or a grid barrier) gave up");
      ++nfin;
      continue;
    }
    const long long used = rc[4 * si] + rc[4 * si + 1];
    s.stats.matcher_calls += s.p.symmetric ? 2 : 1;
    s.stats.block_ncc_evaluated += rc[4 * si + 2];
    if (used == 0) {
      batch_fail(b, s, MIRORR_ENOBLOCKS,
                 "No block matches occurred. Images probably have zero overlap. "
                 "Try supplying a better initial transform.");
      ++nfin;
      continue;
    }
    LtsState hs = rs[si];
    lts_finish(hs);
    s.tfm = hs.tfm;
    if (s.p.symmetric) {
      s.t12f = hs.t12f;
      s.t12b = hs.t12b;
    }
    double cur[12];
    tfm_params(s.tfm, cur);
    const double d = param_delta(s.last, cur, tfm_nparams(s.tfm));
    for (int i = 0; i < 12; ++i) s.last[i] = cur[i];
    ++s.it;
    if (d < 1e-3 || s.it >= std::abs(s.p.iterations)) {
      batch_end_level(s);
      if (s.state == 2) ++nfin;
    }
  }
  if (finished) *finished = nfin;
  b->t_advance += secs(t4, clk::now());
  return MIRORR_OK;
}

}  // namespace

extern "C" {

mirorr_status mirorr_batch_create(mirorr_ctx c, int32_t max_slots, uint64_t hbm_budget,
                                  mirorr_batch *out) {
  if (!c || !out || max_slots < 1 || max_slots > 64) {
    set_error("null argument or max_slots outside 1..64");
    return MIRORR_EINVAL;
  }
  *out = nullptr;
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  mirorr_batch b = new (std::nothrow) mirorr_batch_s;
  if (!b) { set_error("out of host memory"); return MIRORR_ENOMEM; }
  b->c = c;
  b->max_slots = max_slots;
  b->budget = (size_t)hbm_budget;
  b->slots.resize(max_slots);
  const int S = max_slots;
  mirorr_status st = MIRORR_OK;
  if (st == MIRORR_OK) st = b->h_jobs.ensure(sizeof(ResampleJob) * 4 * S);
  if (st == MIRORR_OK) st = b->h_calls.ensure(sizeof(Match16Call) * 2 * S);
  if (st == MIRORR_OK) st = b->h_pf.ensure(sizeof(PfCall) * 2 * S);
  if (st == MIRORR_OK) st = b->h_states.ensure(sizeof(LtsState) * S);
  if (st == MIRORR_OK)
    st = b->h_rd.ensure(sizeof(LtsState) * S + sizeof(long long) * 4 * S + sizeof(unsigned int) * 8 * S);
  if (st == MIRORR_OK) st = b->d_jobs.ensure(sizeof(ResampleJob) * 4 * S);
  if (st == MIRORR_OK) st = b->d_pf.ensure(sizeof(PfCall) * 2 * S);
  if (st == MIRORR_OK) st = b->d_states.ensure(sizeof(LtsState) * S);
  if (st == MIRORR_OK) st = b->d_counts.ensure(sizeof(long long) * 4 * S);
  if (st == MIRORR_OK) st = b->d_ctl.ensure(sizeof(unsigned int) * 8 * S);
  if (st == MIRORR_OK) st = b->d_calls.ensure(sizeof(Match16Call) * 2 * S);
  if (st == MIRORR_OK) st = b->d_lts_args.ensure(lts_args_bytes() * S);
  if (st == MIRORR_OK) st = b->h_lts_args.ensure(lts_args_bytes() * S);
  if (st == MIRORR_OK) st = c->ncc_count.ensure(sizeof(unsigned long long));
  if (st != MIRORR_OK) {
    mirorr_batch_destroy(b);
    return st;
  }
  *out = b;
  return MIRORR_OK;
}

mirorr_status mirorr_batch_destroy(mirorr_batch b) {
  if (!b) return MIRORR_OK;
  cudaSetDevice(b->c->device);
  cudaStreamSynchronize(b->c->stream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (auto &s : b->slots)
    if (s.state) batch_release(b, s);
  for (auto &e : b->pool) cudaFree(e.second);
  b->pool.clear();
  b->pool_bytes = 0;
  HostBuf *hb[] = {&b->h_jobs, &b->h_calls, &b->h_pf, &b->h_states, &b->h_rd, &b->h_lts_args};
  for (HostBuf *x : hb) x->release();
  DevBuf *db[] = {&b->d_jobs, &b->d_pf, &b->d_states, &b->d_counts, &b->d_ctl, &b->d_calls,
                  &b->d_lts_args};
  for (DevBuf *x : db) x->release();
  delete b;
  return MIRORR_OK;
}

mirorr_status mirorr_batch_set_graphs(mirorr_batch b, int32_t on) {
  if (!b) { set_error("null argument"); return MIRORR_EINVAL; }
  b->graphs = on != 0;
  if (!b->graphs && b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return MIRORR_OK;
}

mirorr_status mirorr_batch_submit(mirorr_batch b, const mirorr_geometry *fg, const void *fixed,
                                  const uint8_t *fmask, const mirorr_geometry *mg,
                                  const void *moving, const uint8_t *mmask,
                                  const mirorr_reg_params *p, const mirorr_transform *init,
                                  int64_t *request_id) {
  if (!b || !fg || !mg || !fixed || !moving || !p || !request_id) {
    set_error("null argument");
    return MIRORR_EINVAL;
  }
  mirorr_ctx c = b->c;
  if (!valid_geom(fg) || !valid_geom(mg)) { set_error("invalid image geometry"); return MIRORR_EINVAL; }
  if (!is16(p->storage)) {
    set_error("batched registration stores images in BF16 or F16 (storage %d)", p->storage);
    return MIRORR_EINVAL;
  }
  if (p->kind != KIND_RIGID && p->kind != KIND_AFFINE) {
    set_error("transform kind must be 0 (rigid) or 1 (affine)");
    return MIRORR_EINVAL;
  }
  MB2_TRY(check_bm_params(p->bm));
  if ((p->bm.block_width != 4 && p->bm.block_width != 5) || p->bm.block_gap != 1 ||
      p->bm.nhood_width + p->bm.block_width - 1 > 16) {
    set_error("batched registration needs block width 4 or 5, block gap 1 and a window up to "
              "17 - block width");
    return MIRORR_EINVAL;
  }
  if (!(p->lts_keep > 0.0 && p->lts_keep <= 1.0)) { set_error("lts_keep must lie in (0, 1]"); return MIRORR_EINVAL; }
  if (b->params_set && (p->storage != b->storage || p->bm.nhood_width != b->bm.nhood_width ||
                        p->bm.nhood_gap != b->bm.nhood_gap ||
                        p->bm.block_width != b->bm.block_width)) {
    set_error("the requests of one batch share the storage type, block width, window and block "
              "spacing");
    return MIRORR_EINVAL;
  }
  int si = -1;
  for (int i = 0; i < b->max_slots; ++i)
    if (b->slots[i].state == 0) { si = i; break; }
  if (si < 0) { set_error("no free slot"); return MIRORR_EBUSY; }
  BatchSlot &s = b->slots[si];
  mirorr_reg_params pp = *p;
  if (pp.iterations == 0) pp.iterations = 5;
  if (pp.min_length <= 0) pp.min_length = 32;
  int sched_m[16][3], sched_f[16][3];
  int nl = pyramid_schedule(*fg, *mg, pp.min_length, pp.levels, sched_m, sched_f);
  if (pp.last_level > 0 && pp.last_level < nl) nl = pp.last_level;
  else if (pp.last_level < 0) nl = std::max(1, nl + pp.last_level);
  // the largest level's middle space and block grid size the buffers
  long long max_vox = 0, max_blocks = 0;
  size_t chunk_b = 0, wand_b = 0, stats_b = 0;
  for (int l = 0; l < nl; ++l) {
    mirorr_geometry lf, lm;
    level_geometry(*fg, sched_f[l], lf);
    level_geometry(*mg, sched_m[l], lm);
    int size[3];
    for (int d = 0; d < 3; ++d) size[d] = (int)(((double)lf.size[d] + (double)lm.size[d] + 0.5) / 2.0);
    BmGeom g;
    if (!bm_geometry(size, (int)pp.bm.block_width, (int)pp.bm.block_gap, (int)pp.bm.nhood_gap,
                     (int)pp.bm.nhood_width, g)) {
      set_error("a pyramid level's middle space is smaller than one block");
      return MIRORR_EINVAL;
    }
    Match16Call mc;
    memset(&mc, 0, sizeof(mc));
    prepare16(g, mc);
    max_vox = std::max(max_vox, (long long)size[0] * size[1] * size[2]);
    max_blocks = std::max(max_blocks, g.nblocks);
    chunk_b = std::max(chunk_b, match16_chunk_bytes(mc));
    wand_b = std::max(wand_b, match16_wand_bytes(mc));
    stats_b = std::max(stats_b, match16_stats_bytes(mc));
  }
  const size_t need = slot_bytes(*fg, *mg, pp, fmask != nullptr, mmask != nullptr, max_vox, max_blocks);
  if (need > b->budget) {
    set_error("request needs %zu bytes, more than the whole budget of %zu", need, b->budget);
    return MIRORR_ERANGE;
  }
  if (b->used + need > b->budget) {
    set_error("request needs %zu bytes; %zu of the budget's %zu are in use", need, b->used, b->budget);
    return MIRORR_EBUSY;
  }
  MB2_CUDA_TRY(cudaSetDevice(c->device));
  s = BatchSlot();
  s.p = pp;
  s.fg = *fg;
  s.mg = *mg;
  s.nl = nl;
  memcpy(s.sm, sched_m, sizeof(sched_m));
  memcpy(s.sf, sched_f, sizeof(sched_f));
  s.cap_blocks = max_blocks;
  s.bytes = need;
  b->used += need;
  s.state = 1;  // owns buffers from here (released on failure below)
  const size_t es = elem_size(pp.storage);
  const int ncall = pp.symmetric ? 2 : 1;
  mirorr_status st = MIRORR_OK;
  std::vector<std::pair<DevBuf *, size_t>> bufs;
  auto E = [&](DevBuf &x, size_t n) { bufs.push_back({&x, n}); };
  E(s.in_f, es * vox(fg->size));
  E(s.in_m, es * vox(mg->size));
  if (fmask) E(s.in_fm, vox(fg->size));
  if (mmask) E(s.in_mm, vox(mg->size));
  E(s.lvl_f, sizeof(float) * vox(fg->size));
  E(s.lvl_m, sizeof(float) * vox(mg->size));
  E(s.img_b, es * max_vox);
  E(s.img_s, es * max_vox);
  E(s.msk_b, max_vox);
  E(s.msk_s, max_vox);
  for (int k = 0; k < ncall; ++k) {
    BatchCallBufs &cb = s.call[k];
    E(cb.stats, stats_b);
    E(cb.wand, wand_b);
    E(cb.prep, sizeof(Prep16) * max_blocks);
    E(cb.xs, sizeof(uint32_t) * 64 * max_blocks);
    E(cb.chunked, chunk_b);
    E(cb.fb, sizeof(int) * max_blocks);
    E(cb.best, sizeof(float) * max_blocks);
    E(cb.second, sizeof(float) * max_blocks);
    E(cb.match, sizeof(int32_t) * max_blocks);
    E(cb.status, max_blocks);
    E(cb.tiles, sizeof(unsigned int) * (max_blocks / 2048 + 2));
    if (pp.bm.block_keep < 1.0) {
      E(cb.sel.var, selection_var_bytes(max_blocks));
      E(cb.sel.selected, max_blocks);
      E(cb.sel.select_state, selection_state_bytes());
    }
  }
  E(s.pts_i, sizeof(double) * 3 * ncall * max_blocks);
  E(s.pts_m, sizeof(double) * 3 * ncall * max_blocks);
  E(s.lts_scratch, lts_fit_scratch_bytes(ncall * max_blocks, kLtsCtas));
  st = slot_carve(b, s, bufs);
  if (st == MIRORR_OK) st = upload(c, s.in_f, fixed, es * vox(fg->size));
  if (st == MIRORR_OK) st = upload(c, s.in_m, moving, es * vox(mg->size));
  if (st == MIRORR_OK && fmask) st = upload(c, s.in_fm, fmask, vox(fg->size));
  if (st == MIRORR_OK && mmask) st = upload(c, s.in_mm, mmask, vox(mg->size));
  s.has_fm = fmask != nullptr;
  s.has_mm = mmask != nullptr;
  Tfm t;
  if (st == MIRORR_OK) {
    if (init) {
      if (!from_public(*init, t) || init->kind != pp.kind) {
        set_error("initial transform kind does not match the requested kind");
        st = MIRORR_EINVAL;
      }
    } else {
      double cfix[3], cmov[3], tr[3];
      center_of(*fg, cfix);
      center_of(*mg, cmov);
      tfm_identity(t, pp.kind);
      tfm_set_center(t, cmov);
      for (int d = 0; d < 3; ++d) tr[d] = cfix[d] - cmov[d];
      tfm_set_translation(t, tr);
    }
  }
  if (st != MIRORR_OK) {
    std::string msg = mirorr_last_error();
    batch_release(b, s);
    set_error("%s", msg.c_str());
    return st;
  }
  s.tfm = t;
  tfm_params(t, s.params);
  s.stats.h2d_bytes = (int64_t)(es * (vox(fg->size) + vox(mg->size)) +
                                (fmask ? vox(fg->size) : 0) + (mmask ? vox(mg->size) : 0));
  s.t0 = std::chrono::steady_clock::now();
  s.id = b->next_id++;
  if (!b->params_set) {
    b->params_set = true;
    b->bm = pp.bm;
    b->storage = pp.storage;
  }
  *request_id = s.id;
  return MIRORR_OK;
}

mirorr_status mirorr_batch_step(mirorr_batch b, int32_t *running, int32_t *finished) {
  if (!b) { set_error("null argument"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(b->c->device));
  int r = 0, f = 0;
  mirorr_status st = batch_round(b, &r, &f);
  if (running) *running = r;
  if (finished) *finished = f;
  return st;
}

mirorr_status mirorr_batch_run(mirorr_batch b) {
  if (!b) { set_error("null argument"); return MIRORR_EINVAL; }
  MB2_CUDA_TRY(cudaSetDevice(b->c->device));
  for (int guard = 0; guard < 100000; ++guard) {
    int r = 0, f = 0;
    MB2_TRY(batch_round(b, &r, &f));
    if (r == 0) return MIRORR_OK;
  }
  set_error("batch did not finish");
  return MIRORR_ESTATE;
}

mirorr_status mirorr_batch_poll(mirorr_batch b, int64_t *ids, int32_t capacity, int32_t *n) {
  if (!b || !n) { set_error("null argument"); return MIRORR_EINVAL; }
  int k = 0;
  for (auto &s : b->slots)
    if (s.state == 2 || s.state == 3) {
      if (ids && k < capacity) ids[k] = s.id;
      ++k;
    }
  *n = k;
  return MIRORR_OK;
}

mirorr_status mirorr_batch_result(mirorr_batch b, int64_t id, mirorr_transform *result,
                                  mirorr_reg_stats *stats) {
  if (!b) { set_error("null argument"); return MIRORR_EINVAL; }
  for (auto &s : b->slots) {
    if (s.state == 0 || s.id != id) continue;
    if (s.state == 1) { set_error("request %lld is still running", (long long)id); return MIRORR_ESTATE; }
    cudaSetDevice(b->c->device);
    if (s.state == 3) {
      const mirorr_status st = s.fail;
      const std::string msg = s.fail_msg;
      batch_release(b, s);
      set_error("%s", msg.c_str());
      return st;
    }
    if (result) to_public(s.tfm, *result);
    if (stats) *stats = s.stats;
    batch_release(b, s);
    return MIRORR_OK;
  }
  set_error("no request %lld in the batch", (long long)id);
  return MIRORR_EINVAL;
}

mirorr_status mirorr_batch_cancel(mirorr_batch b, int64_t id) {
  if (!b) { set_error("null argument"); return MIRORR_EINVAL; }
  for (auto &s : b->slots) {
    if (s.state == 0 || s.id != id) continue;
    cudaSetDevice(b->c->device);
    cudaStreamSynchronize(b->c->stream);
    batch_release(b, s);
    return MIRORR_OK;
  }
  set_error("no request %lld in the batch", (long long)id);
  return MIRORR_EINVAL;
}

mirorr_status mirorr_batch_info(mirorr_batch b, int64_t info[8]) {
  if (!b || !info) { set_error("null argument"); return MIRORR_EINVAL; }
  int64_t run = 0, fin = 0;
  for (auto &s : b->slots) {
    if (s.state == 1) ++run;
    if (s.state == 2 || s.state == 3) ++fin;
  }
  info[0] = run;
  info[1] = fin;
  info[2] = (int64_t)b->used;
  info[3] = (int64_t)b->budget;
  info[4] = b->rounds;
  info[5] = b->replays;
  info[6] = b->captures;
  info[7] = b->updates;
  return MIRORR_OK;
}

mirorr_status mirorr_batch_times(mirorr_batch b, double seconds[4]) {
  if (!b || !seconds) { set_error("null argument"); return MIRORR_EINVAL; }
  seconds[0] = b->t_setup;
  seconds[1] = b->t_issue;
  seconds[2] = b->t_device;
  seconds[3] = b->t_advance;
  return MIRORR_OK;
}

}  // extern "C"
