/*
 * mirorr_oracle.c -- CPU restatement of Mirorr's block-matching hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * mirorr_b200/csrc; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  Nothing in the product links or calls it.
 *
 * It restates, in plain C with IEEE double arithmetic and no FMA contraction
 * (built with -ffp-contract=off), the CPU semantics of the reference:
 *
 *   block grid           src/mirorr/itkBlockMatcher.txx:531-600 (ComputeRegionForMatching)
 *                        and itkSparseImageRegionConstIterator.txx:43-88 (raster, x fastest)
 *   variance selection   src/mirorr/itkBlockMatcher.txx:664-719 (dead code, restated with
 *                        a block-keep fraction; cutoff index = (1-keep)*N)
 *   NCC search           src/mirorr/itkBlockMatcher.txx:46-101 (normalizedCorrelation),
 *                        :722-848 (candidate window, clipping, float score buffers,
 *                        best / second-best update)
 *   post-filter          src/mirorr/itkBlockMatcher.txx:850-944 (best > 1e-7 and
 *                        |best - second| > 1e-4)
 *   thread split         src/mirorr/itkBlockMatcherThreaded.txx:97-155 (slabs along the
 *                        largest axis) and :73-89 (output concatenated in thread order)
 *   block -> mm point    src/mirorr/itkAbstractBlockMatcher.h:271-287
 *
 * and the ITK pieces the path calls (ITK is absent here; its published
 * behaviour is restated):
 *   linear resampling    itk::ResampleImageFilter + itk::LinearInterpolateImageFunction
 *                        (call sites itkMirorrRegistrationMethod.txx:523-570,603-604):
 *                        inside test  -0.5 <= c < N-0.5, clamp-to-edge neighbours,
 *                        lerp chain x -> y -> z in double, float output rounded,
 *                        uint8 output clamped to [0,255] and truncated.
 *
 * Parity status: the NCC search of this file is pinned against the
 * reference's own OpenCL kernel (src/mirorr/kernels/optKmatchMask.cl) compiled
 * on the CPU by oracle/build_ref.sh; the remaining pieces (grid, selection,
 * resampler) are restatements with no reference-side golden vectors.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define ORC_API __attribute__((visibility("default")))

static inline long lin3(const int size[3], long x, long y, long z) {
  return (z * (long)size[1] + y) * (long)size[0] + x;
}

/* ------------------------------------------------------------------------ */
/* Block grid: itkBlockMatcher.txx:531-600.  Returns 0 on success, -1 when  */
/* an axis is shorter than a block (the reference computes an unsigned      */
/* underflow there).                                                          */
/* ------------------------------------------------------------------------ */
ORC_API int orc_block_grid(const int size[3], int block_width, int nhood_gap,
                           int nblocks[3], int start[3]) {
  for (int d = 0; d < 3; ++d) {
    if (size[d] < block_width || nhood_gap <= 0) return -1;
    int n = (size[d] - block_width) / nhood_gap + 1;
    int region = nhood_gap * (n - 1) + block_width;
    int gap_at_end = size[d] - region;
    nblocks[d] = n;
    start[d] = gap_at_end / 2;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Dead-code variance of one base block: itkBlockMatcher.txx:690-708.         */
/* Sums run in double in raster order; the square is a float product.        */
/* ------------------------------------------------------------------------ */
static double block_variance(const float *img, const int size[3], const int o[3], int bw) {
  double count = 0, sum = 0, sum_sq = 0;
  for (int z = 0; z < bw; ++z)
    for (int y = 0; y < bw; ++y)
      for (int x = 0; x < bw; ++x) {
        float v = img[lin3(size, o[0] + x, o[1] + y, o[2] + z)];
        count++;
        sum += v;
        float sq = v * v; /* float * float in the reference */
        sum_sq += sq;
      }
  double mean = sum / count;
  return sum_sq / count - mean * mean;
}

ORC_API void orc_block_variances(const float *img, const int size[3], int block_width,
                                 int nhood_gap, double *var_out) {
  int nb[3], st[3];
  if (orc_block_grid(size, block_width, nhood_gap, nb, st)) return;
  long k = 0;
  for (int bz = 0; bz < nb[2]; ++bz)
    for (int by = 0; by < nb[1]; ++by)
      for (int bx = 0; bx < nb[0]; ++bx) {
        int o[3] = {st[0] + bx * nhood_gap, st[1] + by * nhood_gap, st[2] + bz * nhood_gap};
        var_out[k++] = block_variance(img, size, o, block_width);
      }
}

static int cmp_double(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

/* Cutoff of the variance selection (itkBlockMatcher.txx:710-718), with the
 * fraction of blocks KEPT as the knob: index = (unsigned)((1 - keep) * N).
 * keep >= 1 disables the selection (the reference's live behaviour).
 * Returns 1 when the selection is enabled and writes the cutoff. */
ORC_API int orc_variance_cutoff(const double *var, long n, double keep, double *cutoff) {
  if (!(keep < 1.0) || n <= 0) return 0;
  double *s = (double *)malloc(sizeof(double) * (size_t)n);
  memcpy(s, var, sizeof(double) * (size_t)n);
  qsort(s, (size_t)n, sizeof(double), cmp_double);
  unsigned int idx = (unsigned int)((1.0 - keep) * (double)n);
  *cutoff = (idx >= (unsigned long)n) ? s[n - 1] : s[idx];
  free(s);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* normalizedCorrelation: itkBlockMatcher.txx:46-101 (USE_MASK_IN_METRIC).   */
/* ------------------------------------------------------------------------ */
static double ncc_block(const float *base, const float *search, const uint8_t *bmask,
                        const uint8_t *smask, const int size[3], const int bo[3],
                        const int so[3], int bw) {
  double count = 0, mean_s = 0, mean_b = 0;
  for (int z = 0; z < bw; ++z)
    for (int y = 0; y < bw; ++y)
      for (int x = 0; x < bw; ++x) {
        mean_b += base[lin3(size, bo[0] + x, bo[1] + y, bo[2] + z)];
        mean_s += search[lin3(size, so[0] + x, so[1] + y, so[2] + z)];
        count++;
      }
  mean_b /= count;
  mean_s /= count;
  double prod = 0.0, bss = 0.0, sss = 0.0;
  for (int z = 0; z < bw; ++z)
    for (int y = 0; y < bw; ++y)
      for (int x = 0; x < bw; ++x) {
        long bi = lin3(size, bo[0] + x, bo[1] + y, bo[2] + z);
        long si = lin3(size, so[0] + x, so[1] + y, so[2] + z);
        if (!bmask[bi] || !smask[si]) {
          prod += 0.;
          bss += 0.;
          sss += 0.;
        } else {
          double bb = base[bi] - mean_b;
          double sb = search[si] - mean_s;
          prod += bb * sb;
          bss += bb * bb;
          sss += sb * sb;
        }
      }
  if (bss <= 0.0 || sss <= 0.0) return -2.0;
  return prod * prod / bss / sss;
}

typedef struct {
  int block_width, block_gap, nhood_gap, nhood_width;
} orc_params;

/* Candidate window of one block along one axis: itkBlockMatcher.txx:744-756
 * (nhoodEnd is exclusive; the sparse iterator visits start + k*gap < end). */
static void window_axis(int o, int S, const orc_params *p, int *start, int *end) {
  int g = p->block_gap;
  int s = o - (p->nhood_width / 2) * g;
  int e = s + p->nhood_width * g;
  int search_end = S - p->block_width + 1;
  while (s < 0) s += g;
  while (e > search_end) e -= g;
  *start = s;
  *end = e;
}

/* Per-block outputs (grid raster order):
 *   match[3*b]   match origin (voxel index) of the best candidate
 *   best[b], second[b]  float score buffers (USE_FLOAT_SCORE_BUFFER)
 *   status[b]    0 = skipped by the variance selection, 1 = matched
 */
typedef struct {
  const float *base, *search;
  const uint8_t *bmask, *smask;
  int size[3];
  orc_params p;
  int nb[3], st[3];
  const uint8_t *selected; /* NULL = all */
  int32_t *match;
  float *best, *second;
  uint8_t *status;
  /* slab of the block grid handled by this worker */
  int lo[3], hi[3];
} match_job;

static void match_one(const match_job *j, int bx, int by, int bz) {
  long b = ((long)bz * j->nb[1] + by) * j->nb[0] + bx;
  int o[3] = {j->st[0] + bx * j->p.nhood_gap, j->st[1] + by * j->p.nhood_gap,
              j->st[2] + bz * j->p.nhood_gap};
  if (j->selected && !j->selected[b]) {
    j->status[b] = 0;
    return;
  }
  int s0[3], e0[3];
  for (int d = 0; d < 3; ++d) window_axis(o[d], j->size[d], &j->p, &s0[d], &e0[d]);
  float best = -3.0f, second = -3.0f;
  int arg[3] = {s0[0], s0[1], s0[2]};
  int g = j->p.block_gap;
  for (int cz = s0[2]; cz < e0[2]; cz += g)
    for (int cy = s0[1]; cy < e0[1]; cy += g)
      for (int cx = s0[0]; cx < e0[0]; cx += g) {
        int c[3] = {cx, cy, cz};
        double m = ncc_block(j->base, j->search, j->bmask, j->smask, j->size, o, c,
                             j->p.block_width);
        if ((double)best < m) {
          second = best;
          best = (float)m;
          arg[0] = cx; arg[1] = cy; arg[2] = cz;
        } else if ((double)second < m) {
          second = (float)m;
        }
      }
  j->match[3 * b + 0] = arg[0];
  j->match[3 * b + 1] = arg[1];
  j->match[3 * b + 2] = arg[2];
  j->best[b] = best;
  j->second[b] = second;
  j->status[b] = 1;
}

static void *match_worker(void *arg) {
  const match_job *j = (const match_job *)arg;
  for (int bz = j->lo[2]; bz < j->hi[2]; ++bz)
    for (int by = j->lo[1]; by < j->hi[1]; ++by)
      for (int bx = j->lo[0]; bx < j->hi[0]; ++bx) match_one(j, bx, by, bz);
  return NULL;
}

/* Split of the block grid among threads: itkBlockMatcherThreaded.txx:97-155.
 * The split axis is the largest extent of the reduced region
 * (size = G*(n-1)+1 per axis).  Returns the number of slabs used. */
ORC_API int orc_thread_split(const int nb[3], int nhood_gap, int block_width, int threads,
                             int *slab_axis, int *slab_first, int *slab_count) {
  int sz[3];
  for (int d = 0; d < 3; ++d) sz[d] = nhood_gap * (nb[d] - 1) + 1;
  int ax = (sz[0] > sz[1]) ? ((sz[0] > sz[2]) ? 0 : 2) : ((sz[1] > sz[2]) ? 1 : 2);
  *slab_axis = ax;
  /* unsigned arithmetic as in the reference: splitSize - BlockWidth < NhoodGap */
  if ((unsigned)sz[ax] - (unsigned)block_width < (unsigned)nhood_gap) {
    slab_first[0] = 0;
    slab_count[0] = nb[ax];
    return 1;
  }
  unsigned n = (unsigned)(sz[ax] - 1) / (unsigned)nhood_gap + 1;
  unsigned per = n / (unsigned)threads, res = n % (unsigned)threads;
  unsigned used = (per > 0) ? (unsigned)threads : res;
  for (unsigned t = 0; t < used; ++t) {
    unsigned cnt = per + (t < res ? 1 : 0);
    unsigned first = t * per + (t < res ? t : res);
    slab_first[t] = (int)first;
    slab_count[t] = (int)cnt;
  }
  return (int)used;
}

/* Run the matcher over the whole grid with `threads` workers split exactly as
 * the reference's threaded matcher.  Per-block results are written in grid
 * raster order; the reference's thread-order output is rebuilt by
 * orc_emit_points. */
ORC_API int orc_match(const float *base, const float *search, const uint8_t *bmask,
                      const uint8_t *smask, const int size[3], int block_width,
                      int block_gap, int nhood_gap, int nhood_width,
                      const uint8_t *selected, int threads, int32_t *match, float *best,
                      float *second, uint8_t *status) {
  match_job proto;
  memset(&proto, 0, sizeof(proto));
  proto.base = base; proto.search = search; proto.bmask = bmask; proto.smask = smask;
  memcpy(proto.size, size, sizeof(int) * 3);
  proto.p.block_width = block_width; proto.p.block_gap = block_gap;
  proto.p.nhood_gap = nhood_gap; proto.p.nhood_width = nhood_width;
  if (orc_block_grid(size, block_width, nhood_gap, proto.nb, proto.st)) return -1;
  if (block_gap <= 0 || nhood_width <= 0) return -1;
  proto.selected = selected;
  proto.match = match; proto.best = best; proto.second = second; proto.status = status;
  if (threads < 1) threads = 1;
  int axis, first[1024], count[1024];
  if (threads > 1024) threads = 1024;
  int used = orc_thread_split(proto.nb, nhood_gap, block_width, threads, &axis, first, count);
  match_job *jobs = (match_job *)calloc((size_t)used, sizeof(match_job));
  pthread_t *tid = (pthread_t *)calloc((size_t)used, sizeof(pthread_t));
  for (int t = 0; t < used; ++t) {
    jobs[t] = proto;
    for (int d = 0; d < 3; ++d) { jobs[t].lo[d] = 0; jobs[t].hi[d] = proto.nb[d]; }
    jobs[t].lo[axis] = first[t];
    jobs[t].hi[axis] = first[t] + count[t];
  }
  if (used == 1) {
    match_worker(&jobs[0]);
  } else {
    for (int t = 0; t < used; ++t) pthread_create(&tid[t], NULL, match_worker, &jobs[t]);
    for (int t = 0; t < used; ++t) pthread_join(tid[t], NULL);
  }
  free(jobs);
  free(tid);
  return used;
}

/* ITK TransformIndexToPhysicalPoint + half-block offset:
 * itkAbstractBlockMatcher.h:271-287.  direction is row-major. */
static void block_point(const int idx[3], const double origin[3], const double spacing[3],
                        const double direction[9], int bw, double out[3]) {
  double m[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m[3 * r + c] = direction[3 * r + c] * spacing[c];
  for (int r = 0; r < 3; ++r) {
    double v = origin[r];
    for (int c = 0; c < 3; ++c) v += m[3 * r + c] * (double)idx[c];
    out[r] = v;
  }
  double half = 0.5 * (double)bw;
  for (int r = 0; r < 3; ++r) out[r] += spacing[r] * half;
}

/* Post-filter + point emission (itkBlockMatcher.txx:850-944).  order = 0:
 * grid raster order (the OpenCL matcher's order, itkBlockMatcherGPU.txx:441-512);
 * order = T > 0: the threaded CPU matcher's order with T threads.
 * Returns the number of kept blocks; kept_block (optional) receives their
 * grid indices in emission order. */
ORC_API long orc_emit_points(const int size[3], int block_width, int nhood_gap,
                             const int32_t *match, const float *best, const float *second,
                             const uint8_t *status, const double origin[3],
                             const double spacing[3], const double direction[9], int order,
                             double *base_pts, double *match_pts, int64_t *kept_block) {
  int nb[3], st[3];
  if (orc_block_grid(size, block_width, nhood_gap, nb, st)) return -1;
  int axis = 0, first[1024], count[1024], used = 1;
  if (order > 0) {
    if (order > 1024) order = 1024;
    used = orc_thread_split(nb, nhood_gap, block_width, order, &axis, first, count);
  } else {
    first[0] = 0;
    count[0] = nb[0];
    axis = 0;
  }
  long n = 0;
  for (int t = 0; t < used; ++t) {
    int lo[3] = {0, 0, 0}, hi[3] = {nb[0], nb[1], nb[2]};
    lo[axis] = first[t];
    hi[axis] = first[t] + count[t];
    for (int bz = lo[2]; bz < hi[2]; ++bz)
      for (int by = lo[1]; by < hi[1]; ++by)
        for (int bx = lo[0]; bx < hi[0]; ++bx) {
          long b = ((long)bz * nb[1] + by) * nb[0] + bx;
          if (!status[b]) continue;
          double cb = best[b], c2 = second[b];
          if (!(cb > 1e-7)) continue;
          if (!(fabs(cb - c2) > 1e-4)) continue;
          int o[3] = {st[0] + bx * nhood_gap, st[1] + by * nhood_gap, st[2] + bz * nhood_gap};
          int mm[3] = {match[3 * b], match[3 * b + 1], match[3 * b + 2]};
          if (base_pts) block_point(o, origin, spacing, direction, block_width, base_pts + 3 * n);
          if (match_pts) block_point(mm, origin, spacing, direction, block_width, match_pts + 3 * n);
          if (kept_block) kept_block[n] = b;
          ++n;
        }
  }
  return n;
}

/* ------------------------------------------------------------------------ */
/* Linear resampling (ITK ResampleImageFilter + LinearInterpolateImageFunction */
/* restated).  The output-index -> input-continuous-index map is an affine     */
/* map given explicitly: c = e + C[:,0]*i + C[:,1]*j + C[:,2]*k, evaluated     */
/* left to right in double.  Values outside -0.5 <= c < N-0.5 take 0.          */
/* ------------------------------------------------------------------------ */
static double lerp(double a, double b, double t) { return a + (b - a) * t; }

static double interp_at(const float *in, const uint8_t *inm, const int n[3], const double c[3],
                        int *inside) {
  int i0[3], i1[3];
  double t[3];
  for (int d = 0; d < 3; ++d) {
    if (!(c[d] >= -0.5 && c[d] < (double)n[d] - 0.5)) {
      *inside = 0;
      return 0.0;
    }
  }
  *inside = 1;
  for (int d = 0; d < 3; ++d) {
    double f = floor(c[d]);
    int b = (int)f;
    if (b < 0) b = 0;
    double dist = c[d] - (double)b;
    if (dist <= 0.0) dist = 0.0;
    i0[d] = b;
    i1[d] = (b + 1 > n[d] - 1) ? b : b + 1;
    t[d] = dist;
  }
#define V(X, Y, Z) (inm ? (double)inm[lin3(n, X, Y, Z)] : (double)in[lin3(n, X, Y, Z)])
  double v000 = V(i0[0], i0[1], i0[2]), v100 = V(i1[0], i0[1], i0[2]);
  double v010 = V(i0[0], i1[1], i0[2]), v110 = V(i1[0], i1[1], i0[2]);
  double v001 = V(i0[0], i0[1], i1[2]), v101 = V(i1[0], i0[1], i1[2]);
  double v011 = V(i0[0], i1[1], i1[2]), v111 = V(i1[0], i1[1], i1[2]);
#undef V
  double x00 = lerp(v000, v100, t[0]);
  double x10 = lerp(v010, v110, t[0]);
  double x01 = lerp(v001, v101, t[0]);
  double x11 = lerp(v011, v111, t[0]);
  double xx0 = lerp(x00, x10, t[1]);
  double xx1 = lerp(x01, x11, t[1]);
  return lerp(xx0, xx1, t[2]);
}

ORC_API void orc_resample(const float *in, const uint8_t *in_mask, const int in_size[3],
                          const int out_size[3], const double C[9], const double e[3],
                          float *out, uint8_t *out_mask) {
  for (int k = 0; k < out_size[2]; ++k)
    for (int j = 0; j < out_size[1]; ++j)
      for (int i = 0; i < out_size[0]; ++i) {
        double c[3];
        for (int r = 0; r < 3; ++r)
          c[r] = e[r] + C[3 * r + 0] * (double)i + C[3 * r + 1] * (double)j +
                 C[3 * r + 2] * (double)k;
        long o = lin3(out_size, i, j, k);
        int inside;
        if (out) {
          double v = interp_at(in, NULL, in_size, c, &inside);
          out[o] = inside ? (float)v : 0.0f;
        }
        if (out_mask) {
          double v = interp_at(NULL, in_mask, in_size, c, &inside);
          if (!inside) {
            out_mask[o] = 0;
          } else {
            if (v < 0.0) v = 0.0;
            if (v > 255.0) v = 255.0;
            out_mask[o] = (uint8_t)v;
          }
        }
      }
}
