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
  DevBuf select_state;  // selection control block and radix histograms
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
// Work-area sizes of one selection: BmWork::var and BmWork::select_state.
size_t selection_var_bytes(long long nblocks);
size_t selection_state_bytes();
// give_up: a device flag the selection sets when one of its grid-barrier waits
// gives up (the call's result is then invalid), or null.  spin_limit: polls of
// such a wait before it gives up (0: the default, about 0.84 s).
mirorr_status launch_variance_selection(const BmGeom &g, const void *base, double keep,
                                        BmWork &w, const uint8_t **selected_out,
                                        cudaStream_t s, int dtype = MIRORR_DTYPE_F32,
                                        unsigned int *give_up = nullptr,
                                        long long spin_limit = 0);
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

// Per-block base statistics of the 16-bit search.
struct Prep16 {
  float mu;      // mean of the base block (every voxel)
  float sxx;     // sum over base-mask voxels of x~^2 (x~ = x - mu)
  float sxt;     // sum over base-mask voxels of x~
  float sxt_tc;  // sum over every voxel of the two 16-bit parts of x~
  int mmode;     // 1: base mask on everywhere, 2: off everywhere, 0: mixed
  int route;     // 1: the tensor-core search takes the block (else the direct
                 // search's list holds it, or the selection culled it)
  int pad[2];
};

// One matcher call of the 16-bit search: inputs, per-call buffers, outputs
// (filled by the caller) and the geometry and tile layout (prepare16); the
// two tensor-copy descriptors are written by match16_prepare_copies.
struct alignas(64) Match16Call {
  // tensor-copy descriptors (CUtensorMap, 128 bytes each): [0] the window box
  // from the x-chunked copy, [1] the box of the search statistics
  alignas(64) unsigned char tmap[2][128];
  const void *base;
  const uint8_t *bmask;
  const void *search;
  const uint8_t *smask;
  const uint8_t *selected;
  float2 *stats;          // match16_stats_bytes, rows of pitch sp: (mu_y, Syy), Syy sign
                          // bit = footprint leaves the mask
  uint8_t *wand;          // match16_wand_bytes: window-AND passes and per-block flags
  Prep16 *prep;           // nblocks
  uint32_t *xs;           // nblocks x 64 words: the 16-bit parts of the centred base block
  uint4 *chunked;         // match16_chunk_bytes: x-chunked copy of the search image
  float *best;
  float *second;
  int32_t *match;
  uint8_t *status;
  unsigned long long *ncc_count;
  unsigned int *ctl;      // 4 words, zeroed before the launch: [0] tensor blocks,
                          // [1] direct blocks, [2] a bounded wait gave up
  int *fb_list;           // nblocks
  int nx, ny, nz;
  int sp;                 // row pitch of stats (nx rounded up to even: 16-byte rows)
  int nbx, nby, nbz;
  int stx, sty, stz;
  int G, W;
  int bw;                 // block width (4: tensor form possible; 5: direct search only)
  int bpt;                // blocks per tensor tile (G bpt a multiple of 8)
  int tiles_x;
  int chunk_x0, nxc;      // x of the copy's first 8-wide chunk, chunks per row
  int tensor;             // the call takes the tensor form
  int active;             // 0: the launch skips the call
  long long ntiles;
  long long tile0;        // first tile of the call in the launch (set by the launcher)
  long long nblocks;
};
// Geometry and tile layout of a call on block grid g.
void prepare16(const BmGeom &g, Match16Call &c);
size_t match16_chunk_bytes(const Match16Call &c);
size_t match16_wand_bytes(const Match16Call &c);
size_t match16_stats_bytes(const Match16Call &c);
// Writes the tensor-copy descriptors of calls[0, n) (dtype: the storage
// type) from their buffers and geometry.  A replayed graph reads the
// descriptors from the host array at replay, so the caller writes them again
// before every replay (with the tile numbering).
mirorr_status match16_prepare_copies(int dtype, Match16Call *calls, int n);
// Numbers the tensor tiles of calls[0, n) in order (sets each call's tile0)
// and returns their total.  A replayed graph of launch_match16_batch reads the
// descriptors from the host array at replay, so the caller numbers them again
// before every replay.
long long match16_number_tiles(Match16Call *calls, int n);

// Scratch of the 16-bit storage search of one matcher call (tc.cu).
struct Bm16Work {
  DevBuf stats, wand, prep, xs, ctl, fb_list, chunked;
  DevBuf calls;    // device copy of the call descriptors
};
// The 16-bit search of ncalls matcher calls (dtype MIRORR_DTYPE_BF16 or _F16)
// in one launch per stage: box statistics, window-AND, base-block
// preparation, the tensor-core search of every call's tensor tiles in one
// persistent launch, and the direct FP32 search of the blocks the tensor form
// does not take.  host_calls[i].tile0 is set here (match16_number_tiles);
// calls_dev receives the descriptors.  Writes every active call's per-block results.
// every_stage: launch every stage even when no call has tensor tiles (the
// same launch sequence for any set of calls, as a graph update needs).
mirorr_status launch_match16_batch(int dtype, int ncalls, Match16Call *host_calls,
                                   DevBuf &calls_dev, cudaStream_t s, bool every_stage = false);
// One matcher call on 16-bit images with the scratch of w.
mirorr_status launch_match16(int dtype, const BmGeom &g, const void *base, const uint8_t *bmask,
                             const void *search, const uint8_t *smask, const uint8_t *selected,
                             const BmOut &out, Bm16Work &w, unsigned long long *ncc_count,
                             cudaStream_t s);
// True when a bounded wait of the 16-bit search gave up (synchronises).
mirorr_status match16_take_timeout(Bm16Work &w, cudaStream_t s, bool *timed_out);
// Blocks of the last 16-bit search taken by [0] the tensor form, [1] the
// direct search (synchronises).
mirorr_status match16_counts(Bm16Work &w, cudaStream_t s, unsigned int out[2]);

// One matcher call's post-filter in a batch (launch_postfilter_batch): its
// per-block results, grid and point geometry, the compaction tiles (one word
// per 2048 blocks, plus one), the kept-count output and an optional device
// offset added to the output position (the swapped call of a symmetric
// iteration appends after the forward one).
struct PfCall {
  BmOut out;
  BmGeom g;
  PointGeom pg;
  double *pts_b, *pts_m;
  unsigned int *tiles;
  long long *count;
  const long long *offset;
  int active;
};
mirorr_status launch_postfilter_batch(const PfCall *dev_calls, int ncalls, long long max_blocks,
                                      cudaStream_t s);

// Linear resampling with an explicit affine index map (see mirorr_b200.h).
struct ResampleMap {
  double C[9];
  double e[3];
};
// in / out: float32, or 16-bit per in_dtype / out_dtype (MIRORR_DTYPE_*):
// F32 -> F32, F32 -> BF16/F16, and BF16 -> BF16 / F16 -> F16.  A 16-bit output
// is the float result rounded to the storage type.
// mask_ones: in_mask is 255 everywhere (not read; the output mask is 255
// inside the input grid and 0 outside, as its interpolation gives).
mirorr_status launch_resample(const int in_size[3], const void *in, const uint8_t *in_mask,
                              const int out_size[3], const ResampleMap &map, void *out,
                              uint8_t *out_mask, cudaStream_t s, bool nearest = false,
                              int in_dtype = MIRORR_DTYPE_F32, int out_dtype = MIRORR_DTYPE_F32,
                              bool mask_ones = false);
// One pass of launch_resample_batch: float32 image (or none) and uint8 mask
// (or none) on an index map, image output in out_dtype (16-byte aligned),
// mask output 4-byte aligned; inactive jobs are skipped.
struct ResampleJob {
  const float *in;
  const uint8_t *inm;
  void *out;
  uint8_t *outm;
  int in_size[3];
  int out_size[3];
  double C[9];
  double e[3];
  int out_dtype;
  int active;
  int mask_ones;  // inm is 255 everywhere (not read)
};
mirorr_status launch_resample_batch(const ResampleJob *dev_jobs, int njobs, long long max_voxels,
                                    cudaStream_t s);
// BF16 / F16 -> float32 (exact).
mirorr_status launch_from16(const void *in, float *out, long long n, int dtype, cudaStream_t s);
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
  HostBuf out;               // pinned read-back of an uncaptured fit (lts_out_bytes)
};
// A fit in two halves, so that a captured sequence can hold the first: lts_issue
// enqueues the upload of *state_in (after lts_begin), the cooperative launch
// and the read-back of the state, the barrier control and the point counts
// (and *watch_dev when given) into out_host (lts_out_bytes() bytes of host
// memory, pinned when captured; null: the work area's own); lts_collect, after
// the stream has synchronised, takes them into hs (lts_finish applied).
size_t lts_out_bytes();
mirorr_status lts_issue(LtsWork &w, const LtsState *state_in, const double *init_dev,
                        const double *moved_dev, const long long *n_dev, long long n,
                        cudaStream_t st, void *out_host, const unsigned int *watch_dev);
mirorr_status lts_collect(LtsWork &w, const void *out_host, LtsState &hs, int *inner_iters,
                          long long *n_used, unsigned int *watch_host);
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
// The give-up flag ncc_take_timeout reads, allocated (and zeroed) if the
// search has not run yet, for the stages before it.
mirorr_status ncc_give_up_flag(BmWork &w, cudaStream_t s, unsigned int **flag);
// One fit of lts_batch_launch: its state (uploaded after lts_begin), point
// pairs, the two device counters whose sum is the pair count, and scratch of
// lts_fit_scratch_bytes(n_max, ncta) bytes (256-byte aligned).
struct LtsFit {
  LtsState *state;
  const double *init;
  const double *moved;
  const long long *n_dev;
  void *scratch;
};
size_t lts_fit_scratch_bytes(long long n_max, int ncta);
// Bytes of one fit's launch arguments (lts_batch_launch's staging).
size_t lts_args_bytes();
// Runs nfits LTS fits in one cooperative launch, ncta CTAs each (every CTA of
// the launch resident at once); zeroes each fit's barrier and histograms
// first.  args_dev / args_host: argument staging reused across calls.
mirorr_status lts_batch_launch(const LtsFit *fits, int nfits, int ncta, long long spin_limit,
                               DevBuf &args_dev, HostBuf &args_host, cudaStream_t st);
// The device word of a fit's scratch that is non-zero when one of its
// barrier waits gave up.
const int *lts_fit_error_flag(const void *scratch);
// lts_run with every scratch buffer in a static device array sized for
// MIRORR_LTS_NOALLOC_MAX_POINTS pairs: allocates no device memory.  n is the
// number of pairs (no device counters).  Calls on one device must not overlap.
mirorr_status lts_run_noalloc(LtsState &host_state, const double *init_dev,
                              const double *moved_dev, long long n, cudaStream_t s,
                              int *inner_iters);

}  // namespace mb2
