/*
 * mirorr_b200.h -- C ABI of the B200-native Mirorr block-matching registration path.
 *
 * Plain C: opaque handles, plain pointers and sizes, status codes.  No C++
 * exceptions, no torch types.  Every entry point returns mirorr_status; the
 * message of the last failure on the calling thread is mirorr_last_error().
 *
 * Layout conventions (those of itk::Image<float,3> / itk::Image<unsigned char,3>):
 *   volumes are x-fastest, size = {nx, ny, nz}; voxel (x, y, z) sits at
 *   data[(z * ny + y) * nx + x].  Images are float32 (or 16-bit where a
 *   storage type says so, see mirorr_dtype), masks uint8 (0 = outside).
 *   Physical point of index i: origin + direction * diag(spacing) * i,
 *   direction row-major.
 *
 * Threading: a mirorr_ctx and the objects made from it are used from one host
 * thread at a time (the reference's matcher is likewise driven from the
 * single registration thread).  Work is issued on the context's CUDA stream.
 */
#ifndef MIRORR_B200_H
#define MIRORR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MIRORR_ABI_VERSION 2

#if defined(MIRORR_BUILD)
#define MIRORR_API __attribute__((visibility("default")))
#else
#define MIRORR_API
#endif

typedef enum mirorr_status {
  MIRORR_OK = 0,
  MIRORR_EINVAL = 1,     /* bad argument (the reference throws std::out_of_range / runtime_error) */
  MIRORR_ENOMEM = 2,     /* device or host allocation failed */
  MIRORR_ENOBLOCKS = 3,  /* no block matches ("Images probably have zero overlap",
                            itkBlockMatcher.txx:936-943, itkBlockMatcherGPU.txx:505-511) */
  MIRORR_ECUDA = 4,      /* CUDA runtime / launch error, or no usable B200 */
  MIRORR_ETIMEOUT = 5,   /* a bounded device-side wait gave up */
  MIRORR_ESTATE = 6,     /* call out of order (e.g. GetOffsets before images are set) */
  MIRORR_ERANGE = 7,     /* output buffer too small, or a request larger than a limit */
  MIRORR_EBUSY = 8       /* no room now (batch slots or memory budget in use); retry later */
} mirorr_status;

/* Element type of stored volumes.  F32 is the plain path (the drop-in); BF16
 * and F16 store images in 16 bits (round to nearest even from float) and run
 * the block search's cross term on the tensor cores; U8 is the masks' type. */
typedef enum mirorr_dtype {
  MIRORR_DTYPE_F32 = 0,
  MIRORR_DTYPE_BF16 = 1,
  MIRORR_DTYPE_F16 = 2,
  MIRORR_DTYPE_U8 = 3
} mirorr_dtype;

typedef struct mirorr_ctx_s *mirorr_ctx;
typedef struct mirorr_matcher_s *mirorr_matcher;

/* Geometry of a volume (itk::ImageBase: size, spacing, origin, direction). */
typedef struct mirorr_geometry {
  int32_t size[3];
  double spacing[3];
  double origin[3];
  double direction[9]; /* row-major 3x3 */
} mirorr_geometry;

/* Block-matcher parameters: itkAbstractBlockMatcher.h:231-245 (members),
 * defaults itkAbstractBlockMatcher.txx:25-44. */
typedef struct mirorr_bm_params {
  uint32_t block_width;        /* m_BlockWidth: block side in voxels (default 4) */
  uint32_t block_gap;          /* m_BlockGap: candidate stride in voxels (default 1) */
  uint32_t nhood_gap;          /* m_NhoodGap: spacing of the block grid (default 2) */
  uint32_t nhood_width;        /* m_NhoodWidth: candidates per axis, 2R+1 (default 5) */
  double portion_matches_kept; /* m_PortionMatchesKept: 0 -> 0.5, outside [0,1] -> EINVAL
                                  (itkAbstractBlockMatcher.txx:84-100) */
  double block_keep;           /* fraction of blocks kept by base-block variance (the
                                  reference's variance cut-off, itkBlockMatcher.txx:664-719,
                                  which is compiled out there); >= 1 keeps every block */
  int32_t verbosity;           /* m_Verbosity */
} mirorr_bm_params;

/* ---- context ------------------------------------------------------------ */
MIRORR_API mirorr_status mirorr_ctx_create(int32_t device, mirorr_ctx *out);
MIRORR_API mirorr_status mirorr_ctx_destroy(mirorr_ctx ctx);
/* Message of the last failed call on this host thread ("" if none). */
MIRORR_API const char *mirorr_last_error(void);
MIRORR_API int32_t mirorr_abi_version(void);

/* ---- block matcher: replaces itk::AbstractBlockMatcher<ImageType> --------
 * (src/mirorr/itkAbstractBlockMatcher.h:41-313; GPU implementation being
 * replaced: itkBlockMatcherGPU.h/.txx). */
MIRORR_API mirorr_status mirorr_bm_create(mirorr_ctx ctx, mirorr_matcher *out);
MIRORR_API mirorr_status mirorr_bm_destroy(mirorr_matcher m);
/* AbstractBlockMatcher constructor defaults (itkAbstractBlockMatcher.txx:25-44). */
MIRORR_API mirorr_status mirorr_bm_default_params(mirorr_bm_params *p);
/* SetBlockWidth/SetBlockGap/SetNhoodGap/SetNhoodWidth/SetPortionMatchesKept/
 * SetVerbosity (itkAbstractBlockMatcher.h:101-127). */
MIRORR_API mirorr_status mirorr_bm_set_params(mirorr_matcher m, const mirorr_bm_params *p);
/* SetBlockMetricType (itkAbstractBlockMatcher.h:159-163): only "nc" /
 * "normalized_correlation" exists on this path; others -> EINVAL. */
MIRORR_API mirorr_status mirorr_bm_set_metric(mirorr_matcher m, const char *name);
/* SetBaseImage / SetSearchImage (itkAbstractBlockMatcher.txx:45-73): copies
 * host data to device memory owned by the matcher. */
MIRORR_API mirorr_status mirorr_bm_set_base_image(mirorr_matcher m, const mirorr_geometry *g,
                                       const float *host);
MIRORR_API mirorr_status mirorr_bm_set_search_image(mirorr_matcher m, const mirorr_geometry *g,
                                         const float *host);
/* SetBaseMask / SetSearchMask (itkAbstractBlockMatcher.h:87-95); host == NULL
 * restores the default all-255 mask (BeforeGetOffsets, itkBlockMatcher.txx:507-529). */
MIRORR_API mirorr_status mirorr_bm_set_base_mask(mirorr_matcher m, const uint8_t *host);
MIRORR_API mirorr_status mirorr_bm_set_search_mask(mirorr_matcher m, const uint8_t *host);
/* Device-resident variants: the matcher reads caller-owned device memory
 * (no copy); the buffers must stay valid until the next set call. */
MIRORR_API mirorr_status mirorr_bm_set_base_image_device(mirorr_matcher m, const mirorr_geometry *g,
                                              const float *dev);
MIRORR_API mirorr_status mirorr_bm_set_search_image_device(mirorr_matcher m, const mirorr_geometry *g,
                                                const float *dev);
MIRORR_API mirorr_status mirorr_bm_set_base_mask_device(mirorr_matcher m, const uint8_t *dev);
MIRORR_API mirorr_status mirorr_bm_set_search_mask_device(mirorr_matcher m, const uint8_t *dev);
/* No reference counterpart: the element type the matcher stores its images in
 * (MIRORR_DTYPE_F32, the default, or _BF16 / _F16).  Set it before the images;
 * changing it drops the images set so far.  With 16-bit storage the float32
 * setters above convert (round to nearest even) into device copies, the
 * block search runs on the tensor cores (block width 4, block gap 1, window
 * up to 7; other windows up to 13 through a direct FP32 search) and scores
 * are FP32 sums over the stored values rather than the reference's FP64. */
MIRORR_API mirorr_status mirorr_bm_set_storage(mirorr_matcher m, int32_t dtype);
/* 16-bit device images in the storage type (borrowed, no copy). */
MIRORR_API mirorr_status mirorr_bm_set_base_image_device16(mirorr_matcher m, const mirorr_geometry *g,
                                                const void *dev);
MIRORR_API mirorr_status mirorr_bm_set_search_image_device16(mirorr_matcher m,
                                                  const mirorr_geometry *g, const void *dev);
/* SwapImageOrder (itkAbstractBlockMatcher.txx:101-112; the GPU matcher keeps
 * its device buffers, itkBlockMatcherGPU.txx:186-202). */
MIRORR_API mirorr_status mirorr_bm_swap_image_order(mirorr_matcher m);
/* Number of blocks of the current grid (ComputeRegionForMatching,
 * itkBlockMatcher.txx:531-600). */
MIRORR_API mirorr_status mirorr_bm_grid(mirorr_matcher m, int32_t nblocks[3], int32_t start[3]);
/* GetOffsets (itkAbstractBlockMatcher.h:139-146): fills block_positions and
 * match_positions (n x 3 doubles each, mm, blockPositionToPoint convention of
 * itkAbstractBlockMatcher.h:271-287) with the blocks that pass the post-filter,
 * in block-grid raster order.  *n_out receives the count.  If capacity is
 * too small returns ERANGE with *n_out = required count.  Zero kept blocks
 * -> ENOBLOCKS (the GPU matcher's BlockMatcherGPUExceptionAlgo).  ETIMEOUT:
 * a bounded device wait of the search (a tensor copy, or the variance
 * selection's grid barrier) gave up; the whole call's results are invalid. */
MIRORR_API mirorr_status mirorr_bm_get_offsets(mirorr_matcher m, size_t capacity, double *block_positions,
                                    double *match_positions, size_t *n_out);
/* Per-block results of the last GetOffsets, grid raster order, for every
 * block of the grid: match origin voxel index (x,y,z), best and second-best
 * squared NCC, status (0 = culled by the variance selection, 1 = searched,
 * 3 = searched and kept by the post-filter). */
MIRORR_API mirorr_status mirorr_bm_block_results(mirorr_matcher m, size_t capacity, int32_t *match_index,
                                      float *best, float *second, uint8_t *status,
                                      size_t *n_blocks);

/* ---- resampler: itk::ResampleImageFilter + LinearInterpolateImageFunction
 * as wired in itkMirorrRegistrationMethod.txx:523-570,603-604 and
 * itkSymMirorrRegistrationMethod.txx:388-437,481-484.  The output voxel
 * index maps to the input continuous index through c = e + C * idx
 * (C row-major 3x3); outside -0.5 <= c < n - 0.5 the output is 0.  Either
 * image or mask may be NULL.  Host pointers. */
MIRORR_API mirorr_status mirorr_resample(mirorr_ctx ctx, const int32_t in_size[3], const float *in_image,
                              const uint8_t *in_mask, const int32_t out_size[3],
                              const double C[9], const double e[3], float *out_image,
                              uint8_t *out_mask);
/* mirorr_resample (nearest != 0: mirorr_resample_nearest) on device buffers
 * of the context's device: in_image / out_image float32, in_mask / out_mask
 * uint8, either pair may be NULL; out_image 16-byte and out_mask 4-byte
 * aligned.  Issued on the context's stream; returns without waiting for it. */
MIRORR_API mirorr_status mirorr_resample_device(mirorr_ctx ctx, const int32_t in_size[3],
                                     const float *in_image, const uint8_t *in_mask,
                                     const int32_t out_size[3], const double C[9],
                                     const double e[3], float *out_image, uint8_t *out_mask,
                                     int32_t nearest);
/* The same with itk::NearestNeighborInterpolateImageFunction (index
 * floor(c + 0.5)), the final resampling's "nn" interpolator
 * (itkMirorrPyramidImplement.txx:365-479). */
MIRORR_API mirorr_status mirorr_resample_nearest(mirorr_ctx ctx, const int32_t in_size[3],
                                      const float *in_image, const uint8_t *in_mask,
                                      const int32_t out_size[3], const double C[9],
                                      const double e[3], float *out_image, uint8_t *out_mask);
/* Final resampling with itk::BSplineInterpolateImageFunction of order 3, the
 * "bspline" interpolator (and the reference command line's default) of
 * GetInterpolatorFromString / GetResampledImage
 * (itkMirorrPyramidImplement.txx:365-479): FP64 coefficients by the recursive
 * prefilter with mirror boundaries, evaluation on the 4x4x4 support.  Index
 * map and outside value as mirorr_resample.  Image only; host pointers. */
MIRORR_API mirorr_status mirorr_resample_bspline(mirorr_ctx ctx, const int32_t in_size[3],
                                      const float *in_image, const int32_t out_size[3],
                                      const double C[9], const double e[3], float *out_image);
/* The same with itk::WindowedSincInterpolateImageFunction of radius 5 with the
 * Welch window and clamp-to-edge neighbours, the "sinc" interpolator of
 * GetInterpolatorFromString (itkMirorrPyramidImplement.txx:416-425). */
MIRORR_API mirorr_status mirorr_resample_sinc(mirorr_ctx ctx, const int32_t in_size[3],
                                   const float *in_image, const int32_t out_size[3],
                                   const double C[9], const double e[3], float *out_image);
/* Affine index map of the resampler from geometries and a transform
 * y = M x + offset (output grid -> input continuous index). */
MIRORR_API mirorr_status mirorr_resample_map(const mirorr_geometry *out_grid, const mirorr_geometry *in_grid,
                                  const double M[9], const double offset[3], double C[9],
                                  double e[3]);

/* ---- transforms and the LTS fit -------------------------------------------
 * ITK MatrixOffsetTransformBase state: y = matrix * (x - center) + center +
 * translation = matrix * x + offset.  kind: 0 = Euler3DTransform (rigid,
 * params: angles x,y,z (Z*X*Y) + translation), 1 = AffineTransform (params:
 * matrix row-major + translation). */
typedef struct mirorr_transform {
  int32_t kind;
  double matrix[9];
  double offset[3];
  double center[3];
  double params[12];
} mirorr_transform;

/* Classic OptimizeTransform (itkMirorrRegistrationMethod.txx:758-1003):
 * least-trimmed-squares fit of moved ~ T(initial) over n point pairs (mm),
 * composed into *t (m_Transform->Compose(final, true)).  lts_keep replaces the
 * hard-coded 0.5.  *inner_iterations receives the LTS iteration count. */
MIRORR_API mirorr_status mirorr_lts_classic(mirorr_ctx ctx, mirorr_transform *t, size_t n,
                                 const double *initial, const double *moved, double lts_keep,
                                 int32_t *inner_iterations);
/* Symmetric OptimizeTransform(t12F, t12B) (itkSymMirorrRegistrationMethod.txx:729-1442):
 * updates the half-space transforms t12f, t12b and the full transform t. */
MIRORR_API mirorr_status mirorr_lts_symmetric(mirorr_ctx ctx, mirorr_transform *t, mirorr_transform *t12f,
                                   mirorr_transform *t12b, size_t n, const double *initial,
                                   const double *moved, double lts_keep,
                                   int32_t *inner_iterations);

/* No reference counterpart.  The LTS fit of mirorr_lts_classic (t12f and t12b
 * both NULL) or mirorr_lts_symmetric (both non-NULL) on point pairs that are
 * already in device memory on the context's device (initial_dev, moved_dev:
 * n x 3 doubles each, 8-byte aligned), allocating no device memory: its
 * scratch (residuals, radix histograms, per-CTA partial sums, fit state) is
 * one static device array of about 4.2 MB per device, sized for
 * MIRORR_LTS_NOALLOC_MAX_POINTS pairs.  For callers that must not allocate
 * once set up: cudaFree synchronises the whole device, and cudaMalloc fails
 * when another allocator (the caching allocator of a serving process, say)
 * already holds the free memory.  Results equal mirorr_lts_classic /
 * mirorr_lts_symmetric on the same pairs.
 *   - The first call on a device does the set-up: it loads the library's
 *     device code on that device if nothing has yet (which is when the
 *     array's memory is reserved), looks up the array's address and the
 *     cooperative-launch size.  Make that first call early, before a caching
 *     allocator takes the free device memory; later calls reserve nothing.
 *   - n > MIRORR_LTS_NOALLOC_MAX_POINTS returns MIRORR_ERANGE; host pointers,
 *     pointers on another device, and arrays shorter than n x 3 doubles
 *     return MIRORR_EINVAL.
 *   - All calls on one device share the array: calls that overlap in time
 *     (several threads, contexts or streams) race and give wrong results.
 *   - Like the other LTS entry points it copies the fit state in and out
 *     through pageable host memory and synchronises the context's stream
 *     before returning, so it cannot be called while that stream is being
 *     captured into a CUDA graph. */
#define MIRORR_LTS_NOALLOC_MAX_POINTS 524288
MIRORR_API mirorr_status mirorr_lts_noalloc(mirorr_ctx ctx, mirorr_transform *t, mirorr_transform *t12f,
                                 mirorr_transform *t12b, size_t n, const double *initial_dev,
                                 const double *moved_dev, double lts_keep,
                                 int32_t *inner_iterations);

/* ---- registration: MirorrPyramidImplement::RunMirorr over the finest
 * `levels` pyramid levels (itkMirorrPyramidImplement.txx:71-158), classic
 * (itkMirorrRegistrationMethod.txx:422-659) or symmetric
 * (itkSymMirorrRegistrationMethod.txx:238-720) iterations.  Reference CLI
 * equivalents: --reg-mode, -t rigid|affine, --pyr-num L --pyr-end 0, -n,
 * --blockwidth, --blockgap, --nhoodgap, --nhoodwidth, --pyr-min-size. */
typedef struct mirorr_reg_params {
  int32_t symmetric;      /* 0 classic, 1 symmetric (reference default) */
  int32_t kind;           /* 0 rigid (Euler3D), 1 affine */
  int32_t levels;         /* finest pyramid levels to run (0 = all) */
  int32_t iterations;     /* block-matching iterations per level (-n; 0 -> 5) */
  int32_t min_length;     /* --pyr-min-size (default 32) */
  mirorr_bm_params bm;    /* CLI defaults: width 4, gap 1, nhood gap 3, nhood width 7 */
  double lts_keep;        /* LTS keep fraction (reference: 0.5) */
  int32_t verbosity;      /* 1: per-iteration lines; 2: also per-call block routing */
  int32_t last_level;     /* --pyr-end: run the schedule's levels 1..last_level (1 = the
                             coarsest); 0 = all, negative counts back from the finest */
  int32_t storage;        /* element type of the input images and of the middle-space
                             images (mirorr_dtype; no reference counterpart): F32 (the
                             drop-in) or BF16 / F16, whose search runs on the tensor cores */
} mirorr_reg_params;

typedef struct mirorr_reg_stats {
  int32_t levels_run;
  int32_t iterations_run[16];
  int64_t block_ncc_evaluated; /* candidate scores computed (all levels, all calls) */
  int64_t matcher_calls;
  double seconds;              /* host wall time of the call */
  int64_t h2d_bytes;           /* host -> device bytes copied by the call */
  int64_t d2h_bytes;           /* device -> host bytes copied by the call */
} mirorr_reg_stats;

MIRORR_API mirorr_status mirorr_reg_default_params(mirorr_reg_params *p);
/* Full registration from host buffers (the e2e path: uploads inside).  fixed
 * and moving hold elements of p->storage (float32, or 16-bit patterns of
 * BF16 / F16).  Masks may be NULL (all 255).  init may be NULL: centred initialisation
 * (CenteredTransformInitializer GeometryOn, itkMirorrPyramidWrapper.txx:611-623).
 * The result maps moving-image physical points to fixed-image points. */
MIRORR_API mirorr_status mirorr_register(mirorr_ctx ctx, const mirorr_geometry *fixed_geom,
                              const void *fixed, const uint8_t *fixed_mask,
                              const mirorr_geometry *moving_geom, const void *moving,
                              const uint8_t *moving_mask, const mirorr_reg_params *p,
                              const mirorr_transform *init, mirorr_transform *result,
                              mirorr_reg_stats *stats);
/* Same with device-resident inputs (caller-owned device pointers). */
MIRORR_API mirorr_status mirorr_register_device(mirorr_ctx ctx, const mirorr_geometry *fixed_geom,
                                     const void *fixed, const uint8_t *fixed_mask,
                                     const mirorr_geometry *moving_geom, const void *moving,
                                     const uint8_t *moving_mask, const mirorr_reg_params *p,
                                     const mirorr_transform *init, mirorr_transform *result,
                                     mirorr_reg_stats *stats);

/* ---- batched and served registrations ---------------------------------------
 * No reference counterpart (the reference runs one registration per process,
 * mirorr.cxx:93-665).  A batch holds up to max_slots registration requests
 * (BF16 or F16 storage, block width 4 or 5, block gap 1, any block keep; the
 * requests of one batch share the storage type, block width, window and block
 * spacing) on the device at once, within hbm_budget bytes of device memory
 * reserved for them.  Each request is one RunMirorr
 * (itkMirorrPyramidImplement.txx:71-158) with its own size, levels, method and
 * transform kind; its results equal mirorr_register's on the same inputs and
 * parameters up to the order of the LTS fit's floating-point sums.  A step
 * advances every running request by one block-matching iteration with one
 * launch per stage for all of them (the variance selections, the tensor-core
 * search of every request's blocks in one persistent launch, every LTS fit in
 * one cooperative launch).  The step's launches run from a CUDA graph: replayed
 * while the running set and their levels stay unchanged, otherwise updated in
 * place.  Requests may be submitted between steps (continuous batching): a new
 * request starts at its coarsest level while the others continue.  Each
 * request's device buffers live in one allocation; a finished request's
 * allocation is kept for later ones (within the budget), so a running service
 * does not allocate or free device memory per request. */
typedef struct mirorr_batch_s *mirorr_batch;
MIRORR_API mirorr_status mirorr_batch_create(mirorr_ctx ctx, int32_t max_slots,
                                  uint64_t hbm_budget, mirorr_batch *out);
MIRORR_API mirorr_status mirorr_batch_destroy(mirorr_batch b);
/* Admits a request: copies its host inputs (elements of p->storage; masks
 * may be NULL) to the device and reserves its buffers.  MIRORR_EBUSY when no
 * slot is free or its memory does not fit the budget's remainder (retry after
 * results are taken); MIRORR_ERANGE when it would not fit the whole budget;
 * MIRORR_EINVAL for malformed geometry or parameters.  *request_id names it. */
MIRORR_API mirorr_status mirorr_batch_submit(mirorr_batch b, const mirorr_geometry *fixed_geom,
                                  const void *fixed, const uint8_t *fixed_mask,
                                  const mirorr_geometry *moving_geom, const void *moving,
                                  const uint8_t *moving_mask, const mirorr_reg_params *p,
                                  const mirorr_transform *init, int64_t *request_id);
/* One iteration of every running request; *running: requests that took part,
 * *finished: requests that finished (or failed) in this step. */
MIRORR_API mirorr_status mirorr_batch_step(mirorr_batch b, int32_t *running, int32_t *finished);
/* Steps until no request is running. */
MIRORR_API mirorr_status mirorr_batch_run(mirorr_batch b);
/* Ids of finished or failed requests whose results are not taken yet. */
MIRORR_API mirorr_status mirorr_batch_poll(mirorr_batch b, int64_t *ids, int32_t capacity,
                                int32_t *n);
/* A finished request's transform (moving -> fixed physical points) and
 * statistics; frees its slot and memory.  A failed request returns its
 * status (e.g. MIRORR_ENOBLOCKS) and message instead. */
MIRORR_API mirorr_status mirorr_batch_result(mirorr_batch b, int64_t request_id,
                                  mirorr_transform *result, mirorr_reg_stats *stats);
/* Drops a request (running or finished) and frees its slot. */
MIRORR_API mirorr_status mirorr_batch_cancel(mirorr_batch b, int64_t request_id);
/* [0] running, [1] finished and not taken, [2] bytes reserved, [3] budget,
 * [4] steps, [5] steps replayed from a graph, [6] graph instantiations,
 * [7] graph updates in place (a step whose set of requests or levels changed). */
MIRORR_API mirorr_status mirorr_batch_info(mirorr_batch b, int64_t info[8]);
/* Host-clock seconds the batch's steps spent so far: [0] setting up pyramid
 * levels, [1] building the step's descriptors and graph, [2] from launch to
 * the end of the step's device work, [3] advancing the requests. */
MIRORR_API mirorr_status mirorr_batch_times(mirorr_batch b, double seconds[4]);
/* Graph replay of unchanged steps on (default) or off. */
MIRORR_API mirorr_status mirorr_batch_set_graphs(mirorr_batch b, int32_t on);

/* Pyramid schedule (PyramidScheduleTuner::UpdateSymmetric,
 * itkPyramidScheduleTuner.txx:291-414): per level (coarsest first) the
 * shrink factors of the moving and fixed images. */
MIRORR_API mirorr_status mirorr_pyramid_schedule(const mirorr_geometry *fixed_geom,
                                      const mirorr_geometry *moving_geom, int32_t min_length,
                                      int32_t max_levels, int32_t *n_levels,
                                      int32_t moving_factors[16][3],
                                      int32_t fixed_factors[16][3]);
/* One pyramid level of a host volume: separable Gaussian (sigma = f/2 voxels,
 * radius ceil(3 sigma), clamp-to-edge, x then y then z) followed by
 * decimation onto the ITK pyramid grid (spacing * f, size floor(n / f),
 * origin shifted by direction * (spacing_out - spacing_in) / 2) with the
 * linear resampler.  out_geom receives the level geometry. */
MIRORR_API mirorr_status mirorr_pyramid_level(mirorr_ctx ctx, const mirorr_geometry *in_geom,
                                   const float *in_image, const int32_t factors[3],
                                   mirorr_geometry *out_geom, float *out_image,
                                   size_t out_capacity);

/* Timing of the kernels of the last matcher call (CUDA events on the
 * context stream), milliseconds: [0] box statistics, [1] variance selection,
 * [2] NCC search, [3] post-filter + compaction. */
MIRORR_API mirorr_status mirorr_bm_last_timings(mirorr_matcher m, float ms[4]);
/* Diagnostics of the last GetOffsets: [0] candidates re-scored in FP64 by the
 * exact refinement, [1] blocks re-scored entirely in FP64 (refinement list
 * overflow), [2] kept blocks, [3] blocks of the grid, [4] blocks searched by
 * the register-blocked FP32 kernels with a base block inside its mask (window
 * wholly or partly masked), [5] blocks with a partly masked base block (0 for
 * geometries without register-blocked kernels, which search every block with
 * the general kernel).  With 16-bit storage: [0], [1] are 0, [4] blocks searched by
 * the tensor cores, [5] blocks searched by the direct FP32 search. */
MIRORR_API mirorr_status mirorr_bm_last_diagnostics(mirorr_matcher m, int64_t out[6]);
/* Count of kernels launched by this context since creation. */
MIRORR_API int64_t mirorr_ctx_kernel_launches(mirorr_ctx ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events against the library's. */
MIRORR_API void *mirorr_ctx_stream(mirorr_ctx ctx);
/* Iteration graphs of float32 registrations on (default) or off: the first
 * iteration of each pyramid level runs its launches directly, the others
 * replay one CUDA graph of them captured for the level (the same kernels and
 * arithmetic; the transforms and the fit state travel through pinned
 * staging).  Off: every iteration launches directly.  Profiling
 * (mirorr_ctx_set_profiling) and verbosity >= 2 run directly regardless. */
MIRORR_API mirorr_status mirorr_ctx_set_graphs(mirorr_ctx ctx, int32_t on);
/* Per-stage timing of the matcher calls made by registrations: when enabled,
 * CUDA events bracket each stage; mirorr_ctx_stage_times returns the
 * accumulated milliseconds of [box statistics, variance selection, NCC
 * search, post-filter] and the number of matcher calls, and resets them. */
MIRORR_API mirorr_status mirorr_ctx_set_profiling(mirorr_ctx ctx, int32_t on);
MIRORR_API mirorr_status mirorr_ctx_stage_times(mirorr_ctx ctx, double ms[4], int64_t *calls);
/* With profiling on, CUDA events also bracket each launch of the FP32 search
 * kernel for block width 4 (the per-x-lane kernel, the NCC stage's dominant
 * kernel) and a device counter adds up the candidates it scores.  Returns the
 * accumulated milliseconds, launches and candidates, and resets them.  A
 * profiling aid with no counterpart in the reference. */
MIRORR_API mirorr_status mirorr_ctx_search_kernel_times(mirorr_ctx ctx, double *ms, int64_t *launches,
                                             int64_t *candidates);
/* With profiling on, CUDA events also bracket each resampling pass of a
 * registration (an image and its mask into the middle-space grid; one launch
 * when both share an input grid, two otherwise).  Returns the accumulated
 * milliseconds, passes and output voxels, and resets them.  A profiling aid
 * with no counterpart in the reference. */
MIRORR_API mirorr_status mirorr_ctx_resample_times(mirorr_ctx ctx, double *ms, int64_t *passes,
                                        int64_t *voxels);
/* A test aid with no counterpart in the reference: the number of polls a
 * grid-barrier wait of the LTS kernel and of the variance selection makes
 * before it gives up (0 restores the default of 2^23 polls, about 0.84 s).  When a wait gives up, every CTA of the
 * launch returns, the call returns MIRORR_ETIMEOUT, the caller's transforms
 * are left as they were, and the context stays usable.  A tiny limit makes the
 * waits give up on CTAs that are merely late, which is how the tests reach
 * that path without a fault. */
MIRORR_API mirorr_status mirorr_ctx_set_wait_limit(mirorr_ctx ctx, int64_t polls);

#ifdef __cplusplus
}
#endif

#endif /* MIRORR_B200_H */
