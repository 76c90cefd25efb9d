// Internal declarations shared by the libtkb200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tkb200.h"

struct tkb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  size_t smem_optin = 227 * 1024;
  // scratch owned by the context (grown on demand, never shrunk before destroy)
  void *ws = nullptr;
  size_t ws_bytes = 0;
  // device work-queue counters for persistent kernels (zeroed once, self-resetting)
  int *counters = nullptr;
  int64_t launches = 0;
  std::string err;
  cudaGraph_t capturing = nullptr;
  bool in_capture = false;
};

// programmatic dependent launch: a kernel launched with the programmatic-serialization
// attribute may start while the previous kernel of the stream still runs; it must call
// pdl_wait() before touching anything that kernel writes (a no-op without the attribute).
// pdl_trigger() lets the next kernel be scheduled once every CTA of this one has called it.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
#endif

// Launch with programmatic stream serialization: the kernel may start while the previous
// kernel of the stream finishes, so it must call pdl_wait() before its first access to any
// memory that earlier kernels of the stream touch.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// status helpers ------------------------------------------------------------------------
int tkb_set_error(tkb_ctx *ctx, int code, const std::string &msg);
#define TKB_CUDA_TRY(ctx, call)                                                            \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess)                                                                 \
      return tkb_set_error((ctx), TKB_ERR_CUDA,                                            \
                           std::string(#call) + ": " + cudaGetErrorString(_e));            \
  } while (0)

int tkb_ensure_workspace(tkb_ctx *ctx, size_t bytes);

// x[off + i·stride], i < count (count > 0, off, stride ≥ 0) lies inside [0, len): compares
// count − 1 with the room after off instead of forming (count − 1)·stride, which could overflow
inline bool tkb_segment_in_bounds(int64_t off, int64_t count, int64_t stride, int64_t len) {
  if (off >= len) return false;
  return stride == 0 || count - 1 <= (len - 1 - off) / stride;
}

// tree transform ------------------------------------------------------------------------
struct TGroup {
  int32_t ndim;        // canonical dims (after squeezing size-1 dims and merging)
  int32_t da, db;      // tile dims (canonical indices)
  int32_t ta, tb;      // tile extents
  int32_t mode;        // 0 = copy (da fast on both sides), 1 = transpose through smem
  int32_t nouter;
  int32_t outer[TKB_MAX_IND];
  int64_t size[TKB_MAX_IND];
  int64_t ntile_a, ntile_b;
  int64_t task_begin;
  int64_t src_tree_begin, nsrc, dst_tree_begin, ndst, coeff_begin;
  // tree 0 only (single-tree groups): strides of the tile dims a and b, coefficient
  int64_t sa0, sb0, da0, db0;
  double u0;
};

// complete addressing of one task of a single-tree table, resolved on the host (80 bytes)
struct TaskRec {
  int64_t sbase, dbase;      // element offsets of the tile's first element
  int64_t sA, sB, dA, dB;    // strides of the tile dims on both sides
  double u;                  // recoupling coefficient
  int32_t na, nb;            // valid extents of the tile
  int32_t ta, tb;            // tile extents (powers of two; row tiles: ta = na, tb = nb)
  int32_t mode;              // 0: same fastest dim on both sides, 1: transpose
  uint32_t mul;              // row tiles: ⌊(2³²−1)/na⌋ + 1, so e / na = umulhi(e, mul) for e < 2¹⁶
  uint32_t mul2 = 0;         // row tiles copied in pairs: the same for na / 2
  int32_t pairs = 0;         // row tiles: 1 when the rows are contiguous on both sides and every
                             // row starts at an even element, so 16-byte pairs stay aligned
};

struct tkb_table {
  tkb_ctx *owner = nullptr;
  int ngroups = 0;
  int64_t ntasks = 0;
  int64_t elems_read = 0, elems_written = 0;
  int max_trees = 1;             // max(nsrc) over groups
  bool single_tree = false;      // every group has one source and one destination tree
  bool off32 = false;            // every in-tile offset fits 32 bits (both sides)
  size_t smem_f64 = 0;           // dynamic smem bytes needed for f64
  size_t smem_c128 = 0;
  int64_t src_len = 0, dst_len = 0;
  // device arrays
  TGroup *groups = nullptr;
  int64_t *sstr = nullptr, *soff = nullptr, *dstr = nullptr, *doff = nullptr;
  double *coeffs = nullptr;
  int32_t *task_group = nullptr;  // ntasks: the group of every task
  int32_t *task_idx = nullptr;    // ntasks × (2 + TKB_MAX_IND): tile coordinates, outer index
  TaskRec *task_rec = nullptr;    // single-tree tables: per-task bases and extents
  // single-tree tables whose groups all keep their fastest dim (mode 0): exact row tiles
  // (na = the fast extent, not rounded to a power of two) for the register row-copy kernel
  int64_t nrow_tasks = 0;
  TaskRec *row_rec = nullptr;
  int64_t row_pair_elems = 0;     // elements of row tasks that 16-byte pair accesses can copy
};

int tkb_transform_launch(tkb_ctx *ctx, const tkb_table *t, int dtype, void *dst,
                         const void *src, tkb_scalar alpha, tkb_scalar beta, int conj);

// partial trace --------------------------------------------------------------------------
struct TrGroup {
  int64_t dst_off;
  int64_t e_begin, e_end;   // entries of this destination sub-block
  int64_t nelem;            // product of the free sizes
  int64_t task_begin;
  int32_t size[TKB_MAX_IND];
  int64_t dstr[TKB_MAX_IND];
};

struct TrEntry {
  int64_t src_off;
  double coeff;
  int64_t ntr_total;        // product of the traced sizes
  int64_t sstr[TKB_MAX_IND];
  int32_t tsize[TKB_MAX_IND];
  int64_t tstr[TKB_MAX_IND];
};

struct tkb_trace_table {
  tkb_ctx *owner = nullptr;
  int nfree = 0, ntrace = 0;
  int64_t ngroups = 0, ntasks = 0;
  int64_t src_len = 0, dst_len = 0;
  TrGroup *groups = nullptr;
  TrEntry *entries = nullptr;
  int32_t *task_group = nullptr;
};

// grouped gemm --------------------------------------------------------------------------
struct GBlock {
  int64_t m, n, k;
  int64_t offA, offB, offC;
  int64_t lda, ldb, ldc;
  int32_t opA, opB;
  // split precision: workspace offsets of the sliced operands and exponents
  int64_t wsA, wsB, wsEA, wsEB;
  int32_t mpad, npad, kpad;   // padded extents (tile multiples) of the sliced operands
  int32_t skinny;             // 1: n, k ≤ 16 — memory-bound row kernel in every precision
  int32_t fp64only;           // split precision: K too long for two exact int32 pieces — FP64 tiles
};

constexpr int kSkinnyMax = 16;        // n and k bound of the skinny (row-per-thread) path
constexpr int kSkinnyMinRows = 2048;  // smaller blocks go to the tiled kernels
constexpr int kSkinnyRows = 256;       // threads of a skinny CTA (one row each per pass)
constexpr int kSkinnyTaskRows = 1024;  // rows of one skinny task

// CTAs per SM of a kernel (cached per kernel and device; sets the dynamic shared memory limit)
int tkb_occupancy(int device, const void *kfn, int threads, size_t smem);

int tkb_gemm_skinny_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A,
                           const void *B, tkb_scalar alpha, tkb_scalar beta);

struct GTile {
  int32_t block;
  int32_t m0, n0;
  int32_t kind;  // 0 = gemm tile, 1 = β-scale only (k == 0)
};

struct tkb_plan {
  tkb_ctx *owner = nullptr;
  int dtype = 0, precision = 0, slices = 0;
  int64_t nblocks = 0, ntiles = 0;
  GTile *sktasks = nullptr;     // skinny blocks: (block, first row) tasks of kSkinnyTaskRows rows
  int64_t nsk = 0;
  int sk_dim = 0;               // max(n, k) over the skinny blocks
  double flops = 0;
  int64_t lenA = 0, lenB = 0, lenC = 0;
  std::vector<GBlock> hblocks;
  GBlock *blocks = nullptr;
  GTile *tiles = nullptr;
  // split precision
  size_t ws_bytes = 0;          // workspace needed for slices + exponents
  int64_t slice_rows_A = 0, slice_rows_B = 0;  // total padded rows for the slicing pass
  GTile *stiles = nullptr;      // tiles of the split kernel (different tile shape)
  int64_t nstiles = 0;
  int64_t expo_off = 0, expo_bytes = 0;  // exponent region inside the workspace
  void *kstiles = nullptr;      // tcgen05 product tasks (tile, K range, split slot)
  int64_t nkstiles = 0;
  // plain precision: split-K tasks (tile, K range) in a static cost-ordered queue
  void *ptasks = nullptr;
  int64_t nptasks = 0;
  int pgrid = 0;                // CTAs of the plain launch
  double *part = nullptr;       // split-K FP64 partial tiles (rewritten every launch)
  int32_t part_hold0 = 0;       // split: first of the per-CTA hold tiles in `part` (after the partials)
  int *pcnt = nullptr;          // device counters (split-K arrivals; split: claims and readiness too), self-clearing
  unsigned long long *bstat = nullptr;  // split: per-block statistics of the slicing (self-clearing)
  int32_t *bslices = nullptr;   // split: slice count per block of the last launch, then the FP64-checked tiles
  int slices_fixed = 0;         // split: the caller fixed the slice count
  void *sjobs = nullptr;        // slicing tasks (block, operand, rows)
  int64_t nsrows = 0;           // slicing tasks
  int64_t nsctasks = 0;         // of which the first are staged (one CTA each)
  int tile_m = 64, tile_n = 64;
  // split-K knobs (tkb_gemm_plan_create_tuned): pieces per tile at most, K steps per piece at least
  int max_pieces = 8, min_piece_steps = 4;
};

int tkb_gemm_plain_prepare(tkb_ctx *ctx, tkb_plan *p, const std::vector<GTile> &tiles);
int tkb_gemm_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B,
                    tkb_scalar alpha, tkb_scalar beta);
int tkb_gemm_split_prepare(tkb_ctx *ctx, tkb_plan *p);
int tkb_gemm_split_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A,
                          const void *B, tkb_scalar alpha, tkb_scalar beta);

// reductions ----------------------------------------------------------------------------
struct RSeg {
  int64_t off, count, stride;
  double weight;
};

struct tkb_rplan {
  tkb_ctx *owner = nullptr;
  int64_t nseg = 0;
  int64_t total = 0;
  RSeg *segs = nullptr;
  int64_t *seg_begin = nullptr;  // prefix sums of counts (device)
  int nblocks_launch = 0;
};

int tkb_reduce_launch(tkb_ctx *ctx, const tkb_rplan *p, int kind, int dtype, const void *x,
                      const void *y, double *dev_out);
