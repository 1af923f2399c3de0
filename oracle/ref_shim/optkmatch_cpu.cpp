// optkmatch_cpu.cpp -- runs the reference's own OpenCL block-matching kernel
// (src/mirorr/kernels/optKmatchMask.cl, `optKmatch`, lines 67-332) on the CPU.
//
// TEST INFRASTRUCTURE ONLY: this is how the oracle is pinned against the
// reference.  The kernel source is #included unmodified from the reference
// tree (OPTKMATCH_CL is set by oracle/build_ref.sh); this file supplies only
// the OpenCL C built-ins the kernel uses:
//   * work-items are user-level fibers of one OS thread, switched round-robin
//     at every barrier(), which gives barrier() its OpenCL meaning for the
//     uniform control flow of this kernel;
//   * image3d_t reads use the nearest sampler with integer coordinates
//     (itkBlockMatcherGPU.txx:776-781 uploads CL_INTENSITY float / uint8
//     images); reads outside the image return 0 (CLK_ADDRESS_NONE leaves them
//     undefined and the kernel never issues one);
//   * the host side (grid, start offsets, NDRange = nblocks * BlockWidth,
//     local size BlockWidth^3) follows itkBlockMatcherGPU.txx:233-340.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

extern "C" void orc_fiber_switch(void **save_sp, void *load_sp);
asm(R"(
.text
.globl orc_fiber_switch
.type orc_fiber_switch,@function
orc_fiber_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
.size orc_fiber_switch, .-orc_fiber_switch
)");

namespace {

struct Image3D {
  const void *data;
  int w, h, d;
  bool is_u8;
};

struct Float4 { float s0, s1, s2, s3; };
struct UInt4 { unsigned int s0, s1, s2, s3; };
struct Int4 { int x, y, z, w; };

constexpr int kMaxItems = 512;
constexpr size_t kStack = 64 * 1024;

struct GroupRunner {
  int nitems = 0;
  int local_size[3] = {1, 1, 1};
  int group[3] = {0, 0, 0};
  int num_groups[3] = {1, 1, 1};
  int cur = 0;
  int done = 0;
  void *main_sp = nullptr;
  std::vector<void *> sp;
  std::vector<char *> stacks;
  void (*body)(void *) = nullptr;
  void *arg = nullptr;
};

thread_local GroupRunner *tl_runner = nullptr;

void fiber_barrier() {
  GroupRunner *r = tl_runner;
  int me = r->cur;
  int nx = (me + 1) % r->nitems;
  r->cur = nx;
  orc_fiber_switch(&r->sp[me], r->sp[nx]);
}

[[noreturn]] void fiber_main() {
  GroupRunner *r = tl_runner;
  r->body(r->arg);
  int me = r->cur;
  r->done++;
  if (r->done == r->nitems) {
    orc_fiber_switch(&r->sp[me], r->main_sp);
  } else {
    int nx = (me + 1) % r->nitems;
    r->cur = nx;
    orc_fiber_switch(&r->sp[me], r->sp[nx]);
  }
  abort();  // a finished work-item is never resumed
}

void run_group(GroupRunner *r) {
  for (int i = 0; i < r->nitems; ++i) {
    char *top = r->stacks[i] + kStack;
    uintptr_t t = reinterpret_cast<uintptr_t>(top) & ~uintptr_t(15);
    void **s = reinterpret_cast<void **>(t);
    *--s = nullptr;                                        // fake return address
    *--s = reinterpret_cast<void *>(&fiber_main);          // ret target
    for (int k = 0; k < 6; ++k) *--s = nullptr;            // rbp rbx r12-r15
    r->sp[i] = s;
  }
  r->cur = 0;
  r->done = 0;
  orc_fiber_switch(&r->main_sp, r->sp[0]);
}

}  // namespace

// ---- OpenCL C built-ins used by the kernel --------------------------------
typedef Image3D *image3d_t;
typedef int sampler_t;
typedef Float4 float4;
typedef UInt4 uint4;
typedef Int4 int4;
#define __read_only
#define __local
#define CLK_FILTER_NEAREST 1
#define CLK_NORMALIZED_COORDS_FALSE 2
#define CLK_ADDRESS_NONE 4

static inline unsigned int get_local_id(int i) {
  GroupRunner *r = tl_runner;
  int id = r->cur;
  if (i == 0) return id % r->local_size[0];
  if (i == 1) return (id / r->local_size[0]) % r->local_size[1];
  return id / (r->local_size[0] * r->local_size[1]);
}
static inline unsigned int get_group_id(int i) { return tl_runner->group[i]; }
static inline unsigned int get_local_size(int i) { return tl_runner->local_size[i]; }
static inline unsigned int get_num_groups(int i) { return tl_runner->num_groups[i]; }
static inline void barrier(int = 0) { fiber_barrier(); }

static inline Float4 read_imagef(image3d_t img, sampler_t, Int4 p) {
  Float4 v{0.f, 0.f, 0.f, 1.f};
  if (p.x < 0 || p.y < 0 || p.z < 0 || p.x >= img->w || p.y >= img->h || p.z >= img->d) return v;
  size_t o = (static_cast<size_t>(p.z) * img->h + p.y) * img->w + p.x;
  v.s0 = img->is_u8 ? static_cast<float>(static_cast<const uint8_t *>(img->data)[o])
                    : static_cast<const float *>(img->data)[o];
  return v;
}
static inline UInt4 read_imageui(image3d_t img, sampler_t, Int4 p) {
  UInt4 v{0u, 0u, 0u, 1u};
  if (p.x < 0 || p.y < 0 || p.z < 0 || p.x >= img->w || p.y >= img->h || p.z >= img->d) return v;
  size_t o = (static_cast<size_t>(p.z) * img->h + p.y) * img->w + p.x;
  v.s0 = img->is_u8 ? static_cast<const uint8_t *>(img->data)[o]
                    : static_cast<unsigned int>(static_cast<const float *>(img->data)[o]);
  return v;
}

// The kernel file redefines size_t/uint/__kernel/__global for non-OpenCL
// compilers; everything from the standard library is included above.
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wunknown-pragmas"
#pragma GCC diagnostic ignored "-Wunused-variable"
#pragma GCC diagnostic ignored "-Wunused-but-set-variable"
#include OPTKMATCH_CL
#pragma GCC diagnostic pop
#undef size_t
#undef uint

namespace {
struct KernelArgs {
  Image3D *L, *R, *ML, *MR;
  unsigned int *kmatches;
  float *scores, *scores2nd;
  double *rblock, *d1vec;
  unsigned int *m1vec;
  unsigned int w, h, d, bw, nw, pad, bgap, ngap, px, py, pz;
};

void kernel_body(void *p) {
  KernelArgs *a = static_cast<KernelArgs *>(p);
  optKmatch(a->L, a->R, a->ML, a->MR, a->kmatches, a->scores, a->scores2nd, a->rblock,
            a->d1vec, a->m1vec, a->w, a->h, a->d, a->bw, a->nw, a->pad, a->bgap, a->ngap,
            a->px, a->py, a->pz);
}
}  // namespace

// Runs optKmatch over the whole block grid exactly as the OpenCL host does.
// L/ML = base image and mask, R/MR = search image and mask.  Outputs are per
// block in grid raster order: kmatches = linear voxel index of the best match
// origin, scores / scores2nd = best and second-best.  Returns the number of
// blocks, or -1 on invalid arguments.
extern "C" __attribute__((visibility("default"))) long ref_optkmatch(
    const float *L, const float *R, const uint8_t *ML, const uint8_t *MR, int w, int h, int d,
    int block_width, int nhood_width, int block_gap, int nhood_gap, uint32_t *kmatches,
    float *scores, float *scores2nd, int threads) {
  const int bw = block_width;
  const int items = bw * bw * bw;
  if (bw <= 0 || items > kMaxItems || w < bw || h < bw || d < bw || nhood_gap <= 0) return -1;
  int nb[3] = {(w - bw) / nhood_gap + 1, (h - bw) / nhood_gap + 1, (d - bw) / nhood_gap + 1};
  int sz[3] = {w, h, d};
  unsigned int start[3];
  for (int i = 0; i < 3; ++i) {
    int reg = nhood_gap * (nb[i] - 1) + bw;
    unsigned int gap_end = static_cast<unsigned int>(sz[i] - reg);
    start[i] = gap_end / 2;
  }
  long nblocks = static_cast<long>(nb[0]) * nb[1] * nb[2];
  Image3D iL{L, w, h, d, false}, iR{R, w, h, d, false}, iML{ML, w, h, d, true}, iMR{MR, w, h, d, true};
  if (threads < 1) threads = 1;
  auto worker = [&](int tid) {
    GroupRunner r;
    r.nitems = items;
    r.local_size[0] = r.local_size[1] = r.local_size[2] = bw;
    r.num_groups[0] = nb[0]; r.num_groups[1] = nb[1]; r.num_groups[2] = nb[2];
    r.sp.resize(items);
    r.stacks.resize(items);
    for (int i = 0; i < items; ++i) r.stacks[i] = static_cast<char *>(malloc(kStack));
    std::vector<double> rblock(items), d1vec(items);
    std::vector<unsigned int> m1vec(items);
    KernelArgs a{&iL, &iR, &iML, &iMR, kmatches, scores, scores2nd, rblock.data(), d1vec.data(),
                 m1vec.data(), (unsigned)w, (unsigned)h, (unsigned)d, (unsigned)bw,
                 (unsigned)nhood_width, 0u, (unsigned)block_gap, (unsigned)nhood_gap,
                 start[0], start[1], start[2]};
    r.body = kernel_body;
    r.arg = &a;
    tl_runner = &r;
    for (long g = tid; g < nblocks; g += threads) {
      r.group[0] = static_cast<int>(g % nb[0]);
      r.group[1] = static_cast<int>((g / nb[0]) % nb[1]);
      r.group[2] = static_cast<int>(g / (static_cast<long>(nb[0]) * nb[1]));
      run_group(&r);
    }
    tl_runner = nullptr;
    for (int i = 0; i < items; ++i) free(r.stacks[i]);
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(worker, t);
  for (auto &t : pool) t.join();
  return nblocks;
}
