// kernels.cuh -- host-side launchers of the mirorr_b200 CUDA kernels.
#pragma once

#include "common.cuh"
#include "tfm.cuh"

namespace mb2 {

// Geometry of one block-matching call (both images share the grid of the
// base image, as in itkBlockMatcher.txx:734-737).
struct BmGeom {
  int size[3];     // nx, ny, nz
  int nb[3];       // blocks per axis
  int st[3];       // origin of the block grid
  int bw, bgap, ngap, nw;
  long long nblocks;
};

bool bm_geometry(const int size[3], int bw, int bgap, int ngap, int nw, BmGeom &g);

// Scratch needed by one matcher call.
struct BmWork {
  DevBuf stats;     // float2 per voxel of the search image: (mean, masked SS)
  DevBuf var;       // double per block (variance selection)
  DevBuf selected;  // uint8 per block
  DevBuf select_state;
  DevBuf hist;
  DevBuf tiles;     // compaction tile counts/offsets
  DevBuf ncc_lists; // block lists of the NCC stages (general path, fallback)
  DevBuf ncc_ctl;   // NCC counters: [0] general-path blocks, [1] fallback blocks,
                    // [2] FP64-refined candidates, [3] fast-path blocks,
                    // [4] masked-window blocks
  DevBuf ncc_rec;   // per-block FP32 stage results
  DevBuf ncc_bstat; // per-block base statistics
  DevBuf ncc_pad;   // search image with 16-byte aligned rows (when its own are not)
  DevBuf ncc_wand;  // per-block window-AND of the footprint flags (and its passes)
};

struct BmOut {
  float *best;
  float *second;
  int32_t *match;   // linear voxel index of the match origin
  uint8_t *status;  // 0 culled, 1 searched, 3 searched + kept
};

// Per-block points in mm (double3) for base and match blocks.
struct PointGeom {
  double origin[3];
  double a[9];      // direction * diag(spacing), row-major
  double half[3];   // spacing * block_width / 2
};
void point_geom(const double origin[3], const double spacing[3], const double direction[9],
                int bw, PointGeom &pg);

mirorr_status launch_box_stats(const BmGeom &g, const float *search, const uint8_t *smask,
                               float2 *stats, cudaStream_t s);
// base: float32, or 16-bit when dtype is MIRORR_DTYPE_BF16 / _F16.
mirorr_status launch_variance_selection(const BmGeom &g, const void *base, double keep,
                                        BmWork &w, const uint8_t **selected_out,
                                        cudaStream_t s, int dtype = MIRORR_DTYPE_F32);
// ncc_count (optional): device counter incremented by the number of candidate
// scores evaluated.  Profiling (optional): kev[0], kev[1] are recorded around
// the per-x-lane search kernel's launch and xl_count adds up the candidates it
// scores; *xl_ran tells whether that kernel ran.
mirorr_status launch_ncc(const BmGeom &g, const float *base, const uint8_t *bmask,
                         const float *search, const uint8_t *smask, const float2 *stats,
                         const uint8_t *selected, const BmOut &out, BmWork &w,
                         unsigned long long *ncc_count, cudaStream_t s,
                         cudaEvent_t *kev = nullptr, unsigned long long *xl_count = nullptr,
                         bool *xl_ran = nullptr);
// True when a bounded device wait of the NCC stage gave up since the last
// call (then also clears the flag).  Synchronises the stream.
mirorr_status ncc_take_timeout(BmWork &w, cudaStream_t s, bool *timed_out);
// Post-filter (itkBlockMatcher.txx:884-918).  Marks kept blocks (status |= 2),
// counts them into *count_dev and, when pts != nullptr, writes the kept
// blocks' base / match points (mm) in raster order into pts_base / pts_match
// starting at element `pts_offset`.
// offset_dev (optional): device counter added to the output position, so a
// second call can append after a first one without a host round trip.
mirorr_status launch_postfilter(const BmGeom &g, const BmOut &out, BmWork &w,
                                const PointGeom &pg, double *pts_base, double *pts_match,
                                long long *count_dev, const long long *offset_dev,
                                cudaStream_t s);

// Scratch of the 16-bit storage search (tc.cu).
struct Bm16Work {
  DevBuf stats;    // float2 per search position: (mean, Syy), Syy sign bit = footprint leaves the mask
  DevBuf wand;     // window-AND passes and the per-block flags
  DevBuf prep;     // per-block base statistics
  DevBuf xs;       // per-block 16-bit parts of the centred base block
  DevBuf ctl;      // [0] tensor blocks, [1] direct blocks, [2] a bounded wait gave up
  DevBuf fb_list;  // blocks of the direct search
  DevBuf chunked;  // x-chunked copy of the search image for the window tensor copies
};
// One matcher call on 16-bit images (dtype MIRORR_DTYPE_BF16 or _F16): box
// statistics, base-block preparation, the tensor-core search and the direct
// FP32 search of the blocks the tensor form does not take.  Writes `out` for
// every block (the post-filter follows as for the FP32 path).
mirorr_status launch_match16(int dtype, const BmGeom &g, const void *base, const uint8_t *bmask,
                             const void *search, const uint8_t *smask, const uint8_t *selected,
                             const BmOut &out, Bm16Work &w, unsigned long long *ncc_count,
                             cudaStream_t s);
// True when a bounded wait of the 16-bit search gave up (synchronises).
mirorr_status match16_take_timeout(Bm16Work &w, cudaStream_t s, bool *timed_out);
// Blocks of the last 16-bit search taken by [0] the tensor form, [1] the
// direct search (synchronises).
mirorr_status match16_counts(Bm16Work &w, cudaStream_t s, unsigned int out[2]);

// Linear resampling with an explicit affine index map (see mirorr_b200.h).
struct ResampleMap {
  double C[9];
  double e[3];
};
// in / out: float32, or 16-bit per in_dtype / out_dtype (MIRORR_DTYPE_*):
// F32 -> F32, F32 -> BF16/F16, and BF16 -> BF16 / F16 -> F16.  A 16-bit output
// is the float result rounded to the storage type.
mirorr_status launch_resample(const int in_size[3], const void *in, const uint8_t *in_mask,
                              const int out_size[3], const ResampleMap &map, void *out,
                              uint8_t *out_mask, cudaStream_t s, bool nearest = false,
                              int in_dtype = MIRORR_DTYPE_F32, int out_dtype = MIRORR_DTYPE_F32);
// float32 -> BF16 / F16 (round to nearest even).
mirorr_status launch_to16(const float *in, void *out, long long n, int dtype, cudaStream_t s);
// Final-resampling interpolators (interp.cu): cubic B-spline (coef: FP64
// scratch of the input's size) and Welch-windowed sinc of radius 5.
mirorr_status launch_resample_bspline(const int in_size[3], const float *in, const int out_size[3],
                                      const ResampleMap &map, double *coef, float *out,
                                      cudaStream_t s);
mirorr_status launch_resample_sinc(const int in_size[3], const float *in, const int out_size[3],
                                   const ResampleMap &map, float *out, cudaStream_t s);
// Separable Gaussian smoothing along one axis (axis 0 = x).
mirorr_status launch_smooth_axis(const int size[3], const void *in, float *out, int axis,
                                 const double *w, int radius, cudaStream_t s,
                                 int in_dtype = MIRORR_DTYPE_F32);
mirorr_status launch_fill_u8(uint8_t *p, long long n, uint8_t v, cudaStream_t s);

// LTS fit on device (one cooperative launch for the whole inner loop).
struct LtsWork {
  DevBuf state;     // LtsState
  DevBuf resid;     // double per point
  DevBuf partial;   // per-CTA partial sums
  DevBuf hist;      // radix histograms
  DevBuf ctrl;      // barrier + select control
  DevBuf cand;      // candidate keys
  int max_ctas = 0;
  long long spin_limit = 0;  // grid-barrier polls before giving up (0: the default)
};
// n_dev: two device counters whose sum is the number of point pairs; n_max is
// an upper bound used for sizing.  Runs lts_begin / the inner loop /
// lts_finish on host_state.  watch_dev (optional): a device word read back in
// the same synchronisation into *watch_host (the NCC stage's give-up flag).
mirorr_status lts_run(LtsWork &w, LtsState &host_state, const double *init_dev,
                      const double *moved_dev, const long long *n_dev, long long n_max,
                      cudaStream_t s, int *inner_iters, long long *n_used,
                      const unsigned int *watch_dev = nullptr,
                      unsigned int *watch_host = nullptr);
// Window-AND of the footprint-in-mask flags of box statistics (sign bit of
// the second field), per block of g: 1 when every candidate footprint of the
// block's window that lies in the volume is wholly inside the search mask.
mirorr_status launch_window_and(const BmGeom &g, const float2 *stats, DevBuf &buf,
                                const uint8_t **wand, cudaStream_t s);
// The NCC stage's give-up flag (device word), or nullptr before any search.
const unsigned int *ncc_timeout_flag(const BmWork &w);
// lts_run with every scratch buffer in a static device array sized for
// MIRORR_LTS_NOALLOC_MAX_POINTS pairs: allocates no device memory.  n is the
// number of pairs (no device counters).  Calls on one device must not overlap.
mirorr_status lts_run_noalloc(LtsState &host_state, const double *init_dev,
                              const double *moved_dev, long long n, cudaStream_t s,
                              int *inner_iters);

}  // namespace mb2
