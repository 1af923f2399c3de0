// mirorr_main.cpp -- `mirorr`-compatible command line over the C ABI.
//
// Mirrors the reference's option set (src/mirorr/mirorr.cxx:120-275) for the
// block-matching registration this library implements: NIfTI-1 inputs,
// ITK transform files in and out, classic / symmetric, rigid / affine,
// pyramid levels, block parameters, masks, and the final resampled outputs.
// Options of the reference that select machinery outside this path (other
// block metrics, inner resampling modes other than "middle", the experimental
// --reorient-fixed / --reorient-moving identity-space mode) are rejected with a
// message rather than silently changed.
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mirorr_b200.h"
#include "../csrc/tfm.cuh"
#include "nifti_io.hpp"
#include "tfm_io.hpp"

using namespace mirorr_cli;

namespace {

const char *kUsage =
    "Usage: mirorr [options] [moving fixed [last-tfm [start-tfm]]]\n"
    "General:\n"
    "  -m, --moving FILE          moving image (NIfTI-1)\n"
    "  -f, --fixed FILE           fixed image (NIfTI-1)\n"
    "  -l, --last-tfm FILE        output transform, moving to fixed (ITK .tfm)\n"
    "  -s, --start-tfm FILE       initial transform\n"
    "  -t, --tfm-type TYPE        rigid | affine (default rigid)\n"
    "      --reg-mode MODE        classic | symmetric (default symmetric)\n"
    "  -R, --do-not-register      only resample with the given transform\n"
    "      --save-resampled-moving FILE   moving image on the fixed grid\n"
    "      --save-resampled-fixed FILE    fixed image on the moving grid\n"
    "      --final-interpolator I nn | linear | bspline | sinc (default bspline)\n"
    "      --crop mX,mY,fX,fY     crop moving / fixed by voxels on both sides of x and y\n"
    "  -M, --moving-mask FILE     moving image mask\n"
    "  -F, --fixed-mask FILE      fixed image mask\n"
    "  -I, --invert-last-tfm      write the inverse of the result\n"
    "  -i, --invert-start-tfm     invert the initial transform\n"
    "      --fresh                never start from an existing output transform\n"
    "      --echo-cmd             print the command line\n"
    "  -v, --verbose | -q, --quiet | -h, --help\n"
    "Algorithm:\n"
    "  -a, --pyr-start N          first pyramid level (accepted; the schedule starts at 1)\n"
    "  -c, --pyr-end N            last pyramid level, 0 = finest, <0 counts back (default 1)\n"
    "  -d, --pyr-num N            number of pyramid levels (default 1024 = all)\n"
    "  -e, --pyr-min-size N       minimal image dimension of the first level (default 32)\n"
    "  -n, --iterations N         block-matching iterations per level (default 5)\n"
    "      --portion-kept F       portion of matches kept (default 0.5)\n"
    "      --nhoodwidth N         candidates per axis (default 7)\n"
    "      --nhoodgap N           block spacing (default 3)\n"
    "      --blockwidth N         block side (default 4)\n"
    "      --blockgap N           candidate step (default 1)\n"
    "      --blockmetric nc       only normalised correlation\n"
    "  -0, --no-centering-init    start from the identity, not the centred transform\n"
    "      --block-keep F         keep the top F of the blocks by variance (default 1)\n"
    "      --lts-keep F           LTS keep fraction (default 0.5)\n"
    "      --device N             CUDA device (default 0)\n"
    "      --info FILE            print a NIfTI file's ITK geometry (LPS) and exit\n";

struct Args {
  std::map<std::string, std::string> val;
  std::vector<std::string> pos;
  bool has(const std::string &k) const { return val.count(k) != 0; }
  std::string get(const std::string &k, const std::string &d) const {
    auto it = val.find(k);
    return it == val.end() ? d : it->second;
  }
};

Args parse(int argc, char **argv) {
  static const std::map<std::string, std::string> shorts = {
      {"m", "moving"}, {"f", "fixed"}, {"l", "last-tfm"}, {"s", "start-tfm"}, {"t", "tfm-type"},
      {"R", "do-not-register"}, {"M", "moving-mask"}, {"F", "fixed-mask"},
      {"I", "invert-last-tfm"}, {"i", "invert-start-tfm"}, {"v", "verbose"}, {"q", "quiet"},
      {"h", "help"}, {"a", "pyr-start"}, {"c", "pyr-end"}, {"d", "pyr-num"},
      {"e", "pyr-min-size"}, {"n", "iterations"}, {"0", "no-centering-init"}, {"S", "switch-images"}};
  static const char *flags[] = {"do-not-register", "invert-last-tfm", "invert-start-tfm", "verbose",
                                "quiet", "help", "no-centering-init", "fresh", "echo-cmd",
                                "use-gpu-bm", "reorient-fixed", "reorient-moving", "switch-images"};
  static const char *known[] = {
      "moving", "fixed", "last-tfm", "start-tfm", "tfm-type", "reg-mode", "do-not-register",
      "save-reoriented-fixed", "save-reoriented-moving", "save-resampled-fixed",
      "save-resampled-moving", "final-interpolator", "moving-mask", "fixed-mask", "switch-images",
      "invert-last-tfm", "invert-start-tfm", "nthreads", "echo-cmd", "fresh", "help", "verbose",
      "quiet", "pyr-start", "pyr-end", "pyr-num", "pyr-min-size", "resampling-mode", "crop",
      "iterations", "portion-kept", "use-gpu-bm", "reorient-fixed", "reorient-moving", "save-fixed",
      "save-moving", "no-centering-init", "blockmetric", "nhoodwidth", "nhoodgap", "blockwidth",
      "blockgap", "block-keep", "lts-keep", "device", "info"};
  auto is_known = [&](const std::string &k) {
    for (const char *x : known)
      if (k == x) return true;
    return false;
  };
  Args a;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    std::string key;
    if (s.rfind("--", 0) == 0) {
      key = s.substr(2);
      size_t eq = key.find('=');
      if (eq != std::string::npos) {
        if (!is_known(key.substr(0, eq))) throw std::runtime_error("unknown option --" + key.substr(0, eq));
        a.val[key.substr(0, eq)] = key.substr(eq + 1);
        continue;
      }
      if (!is_known(key)) throw std::runtime_error("unknown option " + s);
    } else if (s.size() >= 2 && s[0] == '-' && !(s[1] >= '1' && s[1] <= '9')) {
      auto it = shorts.find(s.substr(1));
      if (it == shorts.end()) throw std::runtime_error("unknown option " + s);
      key = it->second;
    } else {
      a.pos.push_back(s);
      continue;
    }
    bool flag = false;
    for (const char *f : flags)
      if (key == f) flag = true;
    if (flag) {
      a.val[key] = "1";
    } else {
      if (i + 1 >= argc) throw std::runtime_error("option --" + key + " needs a value");
      a.val[key] = argv[++i];
    }
  }
  static const char *posnames[] = {"moving", "fixed", "last-tfm", "start-tfm"};
  for (size_t k = 0; k < a.pos.size(); ++k) {
    if (k >= 4) throw std::runtime_error("too many positional arguments");
    if (!a.has(posnames[k])) a.val[posnames[k]] = a.pos[k];
  }
  return a;
}

void check(mirorr_status s, const char *what) {
  if (s != MIRORR_OK)
    throw std::runtime_error(std::string(what) + ": " + mirorr_last_error());
}

bool exists(const std::string &p) {
  struct stat st;
  return !p.empty() && stat(p.c_str(), &st) == 0;
}

mb2::Tfm to_tfm(const mirorr_transform &t) {
  mb2::Tfm r;
  mb2::tfm_identity(r, t.kind);
  mb2::tfm_set_center(r, t.center);
  mb2::tfm_set_params(r, t.params);
  return r;
}

mirorr_transform from_tfm(const mb2::Tfm &t) {
  mirorr_transform o;
  std::memset(&o, 0, sizeof(o));
  o.kind = t.kind;
  for (int i = 0; i < 9; ++i) o.matrix[i] = t.M[i];
  for (int i = 0; i < 3; ++i) { o.offset[i] = t.off[i]; o.center[i] = t.c[i]; }
  mb2::tfm_params(t, o.params);
  return o;
}

// A transform of the requested kind: a rigid one is widened to affine; an
// affine one cannot be narrowed.
mb2::Tfm as_kind(const mb2::Tfm &t, int kind) {
  if (t.kind == kind) return t;
  if (kind == mb2::KIND_RIGID) throw std::runtime_error("an affine start transform cannot seed a rigid registration");
  mb2::Tfm a;
  mb2::tfm_identity(a, mb2::KIND_AFFINE);
  mb2::tfm_set_center(a, t.c);
  mb2::tfm_set_matrix(a, t.M);
  mb2::tfm_set_translation(a, t.t);
  return a;
}

std::vector<uint8_t> read_mask(const std::string &path, const mirorr_geometry &like) {
  Volume v = read_nifti(path);
  for (int d = 0; d < 3; ++d)
    if (v.geom.size[d] != like.size[d])
      throw std::runtime_error("mask " + path + " does not match its image's size");
  std::vector<uint8_t> m(v.data.size());
  for (size_t i = 0; i < m.size(); ++i) m[i] = v.data[i] != 0.0f ? 255 : 0;
  return m;
}

// Resamples `in` (on grid gin) onto grid gout through y = M x + offset
// (an output physical point maps to an input physical point).
enum class Interp { kNearest, kLinear, kBspline, kSinc };

// GetInterpolatorFromString (itkMirorrPyramidImplement.txx:365-390): the first
// of "nn", "linear", "bspline", "sinc" contained in the name; otherwise
// bspline, with a note.
Interp interpolator_from_string(const std::string &name, bool quiet) {
  if (name.find("nn") != std::string::npos) return Interp::kNearest;
  if (name.find("linear") != std::string::npos) return Interp::kLinear;
  if (name.find("bspline") != std::string::npos) return Interp::kBspline;
  if (name.find("sinc") != std::string::npos) return Interp::kSinc;
  if (!quiet)
    std::printf("Unspecified or unknown interpolator name '%s'. Defaulting to bspline.\n",
                name.c_str());
  return Interp::kBspline;
}

std::vector<float> resample_to(mirorr_ctx ctx, const Volume &in, const mirorr_geometry &gout,
                               const mb2::Tfm &t, Interp interp) {
  double C[9], e[3];
  check(mirorr_resample_map(&gout, &in.geom, t.M, t.off, C, e), "resample map");
  std::vector<float> out((size_t)gout.size[0] * gout.size[1] * gout.size[2]);
  switch (interp) {
    case Interp::kNearest:
      check(mirorr_resample_nearest(ctx, in.geom.size, in.data.data(), nullptr, gout.size, C, e,
                                    out.data(), nullptr), "resample");
      break;
    case Interp::kLinear:
      check(mirorr_resample(ctx, in.geom.size, in.data.data(), nullptr, gout.size, C, e,
                            out.data(), nullptr), "resample");
      break;
    case Interp::kBspline:
      check(mirorr_resample_bspline(ctx, in.geom.size, in.data.data(), gout.size, C, e,
                                    out.data()), "resample");
      break;
    case Interp::kSinc:
      check(mirorr_resample_sinc(ctx, in.geom.size, in.data.data(), gout.size, C, e, out.data()),
            "resample");
      break;
  }
  return out;
}

// OrientImageFilter towards ARI with the image's own direction, which the
// reference applies to both images and both masks before registering
// (itkMirorrPyramidWrapper.txx:79-92, :208-211): every voxel axis is matched
// to the physical axis its direction column points along most (largest
// |component|), and the buffer is permuted and flipped so that axis 0 runs
// along +y (towards posterior), axis 1 along +x (left) and axis 2 along +z
// (superior) in ITK's LPS space.  Spacing, direction columns and origin
// follow, so every voxel keeps its physical position (an oblique direction
// stays oblique).  A direction whose columns share a dominant axis is left
// as it is.
template <class T>
std::vector<T> permute_flip(const std::vector<T> &in, const int32_t n[3], const int p[3],
                            const int f[3]) {
  const int32_t m[3] = {n[p[0]], n[p[1]], n[p[2]]};
  std::vector<T> out(in.size());
  size_t o = 0;
  for (int k = 0; k < m[2]; ++k)
    for (int j = 0; j < m[1]; ++j)
      for (int i = 0; i < m[0]; ++i, ++o) {
        const int ni[3] = {i, j, k};
        long long idx[3];
        for (int a = 0; a < 3; ++a) idx[p[a]] = f[a] > 0 ? ni[a] : m[a] - 1 - ni[a];
        out[o] = in[(size_t)((idx[2] * n[1] + idx[1]) * n[0] + idx[0])];
      }
  return out;
}

void reorient_ari(Volume &v, std::vector<uint8_t> &mask) {
  const double *D = v.geom.direction;
  int dom[3], sgn[3];
  for (int c = 0; c < 3; ++c) {
    int r = 0;
    for (int q = 1; q < 3; ++q)
      if (std::fabs(D[3 * q + c]) > std::fabs(D[3 * r + c])) r = q;
    dom[c] = r;
    sgn[c] = D[3 * r + c] < 0 ? -1 : 1;
  }
  const int target[3] = {1, 0, 2};  // ARI: axis 0 along y, axis 1 along x, axis 2 along z
  int p[3], f[3];
  for (int a = 0; a < 3; ++a) {
    p[a] = -1;
    for (int c = 0; c < 3; ++c)
      if (dom[c] == target[a]) {
        if (p[a] >= 0) return;  // two axes share a dominant direction
        p[a] = c;
      }
    if (p[a] < 0) return;
    f[a] = sgn[p[a]];
  }
  mirorr_geometry g = v.geom;
  double origin[3] = {v.geom.origin[0], v.geom.origin[1], v.geom.origin[2]};
  for (int a = 0; a < 3; ++a) {
    const int c = p[a];
    g.size[a] = v.geom.size[c];
    g.spacing[a] = v.geom.spacing[c];
    for (int r = 0; r < 3; ++r) g.direction[3 * r + a] = f[a] * D[3 * r + c];
    if (f[a] < 0)  // the new first voxel is the old last one along this axis
      for (int r = 0; r < 3; ++r)
        origin[r] += D[3 * r + c] * v.geom.spacing[c] * (double)(v.geom.size[c] - 1);
  }
  for (int r = 0; r < 3; ++r) g.origin[r] = origin[r];
  v.data = permute_flip(v.data, v.geom.size, p, f);
  if (!mask.empty()) mask = permute_flip(mask, v.geom.size, p, f);
  v.geom = g;
}

// CropImageFilter with equal lower and upper crop sizes cx, cy along voxel
// axes 0 and 1 (itkMirorrPyramidWrapper.txx:243-296): the kept voxels keep
// their physical positions.
template <class T>
std::vector<T> crop_xy(const std::vector<T> &in, const int32_t n[3], int cx, int cy) {
  std::vector<T> out;
  out.reserve((size_t)(n[0] - 2 * cx) * (n[1] - 2 * cy) * n[2]);
  for (int k = 0; k < n[2]; ++k)
    for (int j = cy; j < n[1] - cy; ++j)
      for (int i = cx; i < n[0] - cx; ++i)
        out.push_back(in[((size_t)k * n[1] + j) * n[0] + i]);
  return out;
}

void crop_volume(Volume &v, std::vector<uint8_t> &mask, int cx, int cy) {
  if (cx <= 0 && cy <= 0) return;
  cx = cx > 0 ? cx : 0;
  cy = cy > 0 ? cy : 0;
  if (v.geom.size[0] <= 2 * cx || v.geom.size[1] <= 2 * cy)
    throw std::runtime_error("--crop removes the whole image");
  v.data = crop_xy(v.data, v.geom.size, cx, cy);
  if (!mask.empty()) mask = crop_xy(mask, v.geom.size, cx, cy);
  const double *D = v.geom.direction;
  for (int r = 0; r < 3; ++r)
    v.geom.origin[r] += D[3 * r] * v.geom.spacing[0] * cx + D[3 * r + 1] * v.geom.spacing[1] * cy;
  v.geom.size[0] -= 2 * cx;
  v.geom.size[1] -= 2 * cy;
}

int run(int argc, char **argv) {
  Args a = parse(argc, argv);
  if (a.has("help") || argc == 1) {
    std::fputs(kUsage, stdout);
    return 0;
  }
  if (a.has("info")) {
    const Volume v = read_nifti(a.get("info", ""));
    const mirorr_geometry &g = v.geom;
    std::printf("size %d %d %d\nspacing %.9g %.9g %.9g\norigin %.9g %.9g %.9g\ndirection",
                g.size[0], g.size[1], g.size[2], g.spacing[0], g.spacing[1], g.spacing[2],
                g.origin[0], g.origin[1], g.origin[2]);
    for (int i = 0; i < 9; ++i) std::printf(" %.9g", g.direction[i]);
    double s = 0.0;
    for (float x : v.data) s += x;
    std::printf("\nsum %.9g\n", s);
    // the geometry the registration sees (reoriented to ARI) and its first voxel
    Volume r = v;
    std::vector<uint8_t> none;
    reorient_ari(r, none);
    const mirorr_geometry &h = r.geom;
    std::printf("ari_size %d %d %d\nari_spacing %.9g %.9g %.9g\nari_origin %.9g %.9g %.9g\n"
                "ari_direction", h.size[0], h.size[1], h.size[2], h.spacing[0], h.spacing[1],
                h.spacing[2], h.origin[0], h.origin[1], h.origin[2]);
    for (int i = 0; i < 9; ++i) std::printf(" %.9g", h.direction[i]);
    std::printf("\nari_first %.9g %.9g\n", r.data.front(), r.data.back());
    return 0;
  }
  const bool quiet = a.has("quiet"), verbose = a.has("verbose");
  if (a.has("echo-cmd")) {
    for (int i = 0; i < argc; ++i) std::printf("%s%s", i ? " " : "", argv[i]);
    std::printf("\n");
  }
  for (const char *k : {"reorient-fixed", "reorient-moving", "save-fixed", "save-moving",
                        "save-reoriented-fixed", "save-reoriented-moving", "switch-images"})
    if (a.has(k)) throw std::runtime_error(std::string("--") + k + " is not available in this command line (not part of the registration path it implements)");
  if (a.get("blockmetric", "nc") != "nc")
    throw std::runtime_error("only the normalised correlation block metric (nc) is available");
  if (a.get("resampling-mode", "middle") != "middle")
    throw std::runtime_error("only the middle inner resampling mode is available");
  const Interp interp = interpolator_from_string(a.get("final-interpolator", "bspline"), quiet);
  if (!a.has("moving") || !a.has("fixed")) throw std::runtime_error("moving and fixed images are required");

  const std::string tt = a.get("tfm-type", "rigid");
  int kind;
  if (tt == "rigid" || tt == "quat") kind = mb2::KIND_RIGID;
  else if (tt == "affine") kind = mb2::KIND_AFFINE;
  else throw std::runtime_error("unknown transform type " + tt);
  const std::string mode = a.get("reg-mode", "symmetric");
  if (mode != "classic" && mode != "symmetric") throw std::runtime_error("unknown registration mode " + mode);

  Volume moving = read_nifti(a.get("moving", ""));
  Volume fixed = read_nifti(a.get("fixed", ""));
  std::vector<uint8_t> mmask, fmask;
  if (!a.get("moving-mask", "").empty()) mmask = read_mask(a.get("moving-mask", ""), moving.geom);
  if (!a.get("fixed-mask", "").empty()) fmask = read_mask(a.get("fixed-mask", ""), fixed.geom);

  // the CUDA context, created when registration or resampling needs it
  mirorr_ctx ctx = nullptr;
  auto context = [&]() {
    if (!ctx) check(mirorr_ctx_create(std::atoi(a.get("device", "0").c_str()), &ctx), "CUDA context");
    return ctx;
  };

  // initial transform: start-tfm, else an existing output (unless --fresh)
  const std::string last = a.get("last-tfm", ""), start = a.get("start-tfm", "");
  bool have_init = false;
  mb2::Tfm init;
  std::string init_from = start;
  if (init_from.empty() && !a.has("fresh") && exists(last)) init_from = last;
  if (!init_from.empty()) {
    init = to_tfm(read_tfm(init_from));
    if (a.has("invert-start-tfm")) {
      mb2::Tfm inv;
      if (!mb2::tfm_inverse(init, inv)) throw std::runtime_error("start transform is singular");
      init = inv;
    }
    init = as_kind(init, kind);
    have_init = true;
  } else if (a.has("no-centering-init")) {
    mb2::tfm_identity(init, kind);
    have_init = true;
  }

  // the images the registration sees: reoriented to ARI, then cropped; the
  // final resampling uses the inputs as read (GetResampledImage is given
  // fixedImage_in / movingImage_in, itkMirorrPyramidWrapper.txx:745,801)
  Volume reg_moving = moving, reg_fixed = fixed;
  std::vector<uint8_t> reg_mmask = mmask, reg_fmask = fmask;
  reorient_ari(reg_moving, reg_mmask);
  reorient_ari(reg_fixed, reg_fmask);
  if (a.has("crop") && !a.get("crop", "").empty()) {
    int c[4] = {0, 0, 0, 0};
    if (std::sscanf(a.get("crop", "").c_str(), "%d,%d,%d,%d", &c[0], &c[1], &c[2], &c[3]) != 4)
      throw std::runtime_error("--crop takes movingX,movingY,fixedX,fixedY");
    crop_volume(reg_moving, reg_mmask, c[0], c[1]);
    crop_volume(reg_fixed, reg_fmask, c[2], c[3]);
  }

  mb2::Tfm result = init;
  if (!a.has("do-not-register")) {
    mirorr_reg_params p;
    check(mirorr_reg_default_params(&p), "parameters");
    p.symmetric = mode == "symmetric";
    p.kind = kind;
    p.levels = std::atoi(a.get("pyr-num", "1024").c_str());
    if (p.levels >= 16) p.levels = 0;  // as many as the schedule makes
    p.last_level = std::atoi(a.get("pyr-end", "1").c_str());
    p.iterations = std::atoi(a.get("iterations", "0").c_str());
    p.min_length = std::atoi(a.get("pyr-min-size", "32").c_str());
    p.bm.block_width = (uint32_t)std::atoi(a.get("blockwidth", "4").c_str());
    p.bm.block_gap = (uint32_t)std::atoi(a.get("blockgap", "1").c_str());
    p.bm.nhood_gap = (uint32_t)std::atoi(a.get("nhoodgap", "3").c_str());
    p.bm.nhood_width = (uint32_t)std::atoi(a.get("nhoodwidth", "7").c_str());
    p.bm.portion_matches_kept = std::atof(a.get("portion-kept", "0.5").c_str());
    p.bm.block_keep = std::atof(a.get("block-keep", "1").c_str());
    p.lts_keep = std::atof(a.get("lts-keep", "0.5").c_str());
    p.verbosity = verbose ? 1 : 0;
    mirorr_transform init_pub = from_tfm(init), res;
    mirorr_reg_stats st;
    check(mirorr_register(context(), &reg_fixed.geom, reg_fixed.data.data(),
                          reg_fmask.empty() ? nullptr : reg_fmask.data(), &reg_moving.geom,
                          reg_moving.data.data(), reg_mmask.empty() ? nullptr : reg_mmask.data(),
                          &p, have_init ? &init_pub : nullptr, &res, &st),
          "registration");
    result = to_tfm(res);
    if (!quiet) {
      std::printf("mirorr: %s %s registration, %d level(s), %.3f s\n", mode.c_str(), tt.c_str(),
                  st.levels_run, st.seconds);
    }
  } else if (!have_init) {
    throw std::runtime_error("--do-not-register needs a transform (start-tfm or last-tfm)");
  }

  if (!last.empty() && (!a.has("do-not-register") || last != init_from)) {
    mb2::Tfm out = result;
    if (a.has("invert-last-tfm")) {
      if (!mb2::tfm_inverse(result, out)) throw std::runtime_error("result transform is singular");
    }
    write_tfm(last, from_tfm(out));
    if (!quiet) std::printf("mirorr: wrote %s\n", last.c_str());
  }
  // final resampling: the transform maps moving points to fixed points
  if (a.has("save-resampled-moving")) {
    mb2::Tfm inv;
    if (!mb2::tfm_inverse(result, inv)) throw std::runtime_error("transform is singular");
    std::vector<float> out = resample_to(context(), moving, fixed.geom, inv, interp);
    write_nifti_float(a.get("save-resampled-moving", ""), fixed.geom, out.data());
  }
  if (a.has("save-resampled-fixed")) {
    std::vector<float> out = resample_to(context(), fixed, moving.geom, result, interp);
    write_nifti_float(a.get("save-resampled-fixed", ""), moving.geom, out.data());
  }
  if (ctx) mirorr_ctx_destroy(ctx);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "mirorr: %s\n", e.what());
    return 1;
  }
}
