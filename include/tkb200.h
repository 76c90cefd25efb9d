/*
 * tkb200.h — C ABI of libtkb200.so, the B200 (sm_100a) kernels behind TensorKit's
 * symmetric-contraction path.
 *
 * The library only sees flat device vectors (the `data` field of a TensorMap with
 * CuVector storage), flattened tree-transformer tables and per-block GEMM descriptors.
 * Every export returns an int status (TKB_OK = 0); nothing throws across the ABI.
 * All launches are asynchronous on the context's stream. Device pointers are borrowed
 * for the duration of the call (until stream completion); tables, plans and graphs are
 * owned by the library and released with the matching *_destroy call.
 *
 * Reference interfaces replaced (paths inside TensorKit.jl v0.17.1):
 *   tkb_treetransform   <- add_transform_kernel!(data_dst::DenseVector, data_src::DenseVector,
 *                          p, transformer::{Abelian,Generic}TreeTransformer, α, β, ...)
 *                          src/tensors/indexmanipulations.jl:658-726
 *   tkb_table_create    <- AbelianTreeTransformer / GenericTreeTransformer construction and
 *                          treebraider caching, src/tensors/treetransformers.jl:10-120,156-167
 *   tkb_grouped_gemm    <- LinearAlgebra.mul!(tC, tA, tB, α, β) blockwise loop,
 *                          src/tensors/linalg.jl:330-370
 *   tkb_reduce          <- norm (src/tensors/linalg.jl:257-282), tr (linalg.jl:319-327),
 *                          inner (src/tensors/vectorinterface.jl:114-130)
 *   tkb_graph_*         <- replay of TO.tensorcontract! sequences of one @tensor network,
 *                          src/tensors/tensoroperations.jl:130-161,392-462
 */
#ifndef TKB200_H
#define TKB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TKB_MAX_IND 8

enum tkb_status {
  TKB_OK = 0,
  TKB_ERR_ARG = 1,         /* invalid argument / null handle (ArgumentError) */
  TKB_ERR_SIZE = 2,        /* table or descriptor addresses outside the data (SpaceMismatch) */
  TKB_ERR_OOM = 3,         /* device allocation failed */
  TKB_ERR_CUDA = 4,        /* a CUDA runtime call failed */
  TKB_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
  TKB_ERR_UNSUPPORTED = 6  /* configuration not supported by this build */
};

enum tkb_dtype { TKB_F64 = 0, TKB_C128 = 1 };
enum tkb_precision { TKB_PLAIN = 0, TKB_SPLIT_INT8 = 1 };
enum tkb_op { TKB_OP_N = 0, TKB_OP_T = 1, TKB_OP_C = 2 };
enum tkb_reduce_kind { TKB_NORM2 = 0, TKB_INNER = 1, TKB_TRACE = 2 };

typedef struct tkb_scalar { double re, im; } tkb_scalar;

typedef struct tkb_ctx tkb_ctx;
typedef struct tkb_table tkb_table;
typedef struct tkb_plan tkb_plan;
typedef struct tkb_rplan tkb_rplan;
typedef struct tkb_graph tkb_graph;

/* ---- context ------------------------------------------------------------------------ */
int tkb_version(void);
/* stream: a cudaStream_t (0 = legacy default stream). workspace_bytes: scratch held by
 * the context for split-precision operands and reduction partials (grown on demand). */
int tkb_ctx_create(int device, void *stream, size_t workspace_bytes, tkb_ctx **out);
int tkb_ctx_destroy(tkb_ctx *ctx);
int tkb_ctx_set_stream(tkb_ctx *ctx, void *stream);
/* Waits for the context's stream. Returns TKB_ERR_TIMEOUT (and clears the record) when a
 * bounded device wait of an earlier launch on this context gave up; tkb_last_error names it. */
int tkb_ctx_synchronize(tkb_ctx *ctx);
/* Diagnostic (no counterpart in the reference): launches one kernel that waits on a device
 * flag that nothing sets, for at most timeout_us microseconds (1 .. 1000000), and records the
 * timeout like any bounded device wait of the library; the next tkb_ctx_synchronize reports
 * TKB_ERR_TIMEOUT and the context stays usable. It exercises the error path of the bounded
 * waits without faulting the GPU. */
int tkb_selftest_bounded_wait(tkb_ctx *ctx, int64_t timeout_us);
/* kernels launched by this context since creation (for launch accounting) */
int tkb_ctx_launch_count(const tkb_ctx *ctx, int64_t *count);
const char *tkb_last_error(const tkb_ctx *ctx);

/* ---- tree-transform tables ---------------------------------------------------------- */
/* A flattened AbelianTreeTransformer (one tree per group, U = [[coeff]]) or
 * GenericTreeTransformer (one group per fusion block, U rows = destination trees).
 * All arrays are host pointers, offsets are 0-based element offsets, strides in elements.
 * perm[k] (0-based) is the source dimension that becomes destination dimension k. */
typedef struct tkb_table_desc {
  int32_t nind;
  int32_t perm[TKB_MAX_IND];
  int64_t ngroups;
  const int64_t *group_src_ptr;  /* ngroups+1: prefix sums of source trees per group */
  const int64_t *group_dst_ptr;  /* ngroups+1: prefix sums of destination trees per group */
  const int64_t *coeff_ptr;      /* ngroups+1: prefix sums of rows*cols */
  const double *coeffs;          /* row-major U blocks */
  const int64_t *sizes;          /* ngroups*nind: source sub-block sizes */
  const int64_t *src_strides;    /* ntrees_src*nind */
  const int64_t *src_offsets;    /* ntrees_src */
  const int64_t *dst_strides;    /* ntrees_dst*nind (destination dim order) */
  const int64_t *dst_offsets;    /* ntrees_dst */
  int64_t src_len;               /* elements in the source data vector */
  int64_t dst_len;               /* elements in the destination data vector */
} tkb_table_desc;

int tkb_table_create(tkb_ctx *ctx, const tkb_table_desc *desc, tkb_table **out);
int tkb_table_destroy(tkb_table *table);
/* number of CTA tasks and algorithmic elements read/written per call (β = 0) */
int tkb_table_info(const tkb_table *table, int64_t *ntasks, int64_t *elems_read,
                   int64_t *elems_written);

/* dst = β·dst + α·Σ_j U_ij · permute(src_j, perm), per destination sub-block i.
 * conj_src != 0 reads the source with complex conjugation (lazy adjoint source). */
int tkb_treetransform(tkb_ctx *ctx, const tkb_table *table, int dtype, void *dst,
                      const void *src, tkb_scalar alpha, tkb_scalar beta, int conj_src);

/* ---- partial-trace tables ------------------------------------------------------------ */
/* Flattened trace_permute! (src/tensors/tensoroperations.jl:212-296): one group per
 * destination sub-block (every sub-block of the destination, so that β reaches all of
 * them); its entries are the source sub-blocks whose permuted trees split into it, with the
 * recoupling coefficient times dim(g.coupled)/dim(g.uncoupled[1]).
 *   dst_g[x] = β·dst_g[x] + α·Σ_e coeff_e · Σ_t src[off_e + Σ_k x_k·str_e,k + Σ_l t_l·tstr_e,l]
 * x runs over the group's free sizes (destination order), t over the entry's traced sizes,
 * tstr_e,l = stride(q₁[l]) + stride(q₂[l]) of the source sub-block. */
typedef struct tkb_trace_desc {
  int32_t nfree;                 /* free legs, ≤ TKB_MAX_IND */
  int32_t ntrace;                /* traced leg pairs, 1..TKB_MAX_IND */
  int64_t ngroups;
  const int64_t *group_entry_ptr;  /* ngroups+1: prefix sums of entries per group */
  const int64_t *sizes;            /* ngroups*nfree: free sizes */
  const int64_t *dst_strides;      /* ngroups*nfree */
  const int64_t *dst_offsets;      /* ngroups */
  const int64_t *src_strides;      /* nentries*nfree: source strides of the free legs */
  const int64_t *trace_sizes;      /* nentries*ntrace */
  const int64_t *trace_strides;    /* nentries*ntrace */
  const int64_t *src_offsets;      /* nentries */
  const double *coeffs;            /* nentries */
  int64_t src_len, dst_len;        /* elements in the data vectors (bounds check) */
} tkb_trace_desc;

typedef struct tkb_trace_table tkb_trace_table;
/* replaces the per-sub-block TO.tensortrace! calls of _trace_permute!
 * (src/tensors/tensoroperations.jl:246-296) with one table built once per structure */
int tkb_trace_table_create(tkb_ctx *ctx, const tkb_trace_desc *desc, tkb_trace_table **out);
int tkb_trace_table_destroy(tkb_trace_table *table);
/* conj_src != 0 reads the source with complex conjugation (lazy adjoint source) */
int tkb_tracetransform(tkb_ctx *ctx, const tkb_trace_table *table, int dtype, void *dst,
                       const void *src, tkb_scalar alpha, tkb_scalar beta, int conj_src);

/* ---- grouped block GEMM ------------------------------------------------------------- */
/* C_b = α·op(A_b)·op(B_b) + β·C_b for every block b; column-major blocks in flat vectors.
 * op(A_b) is m×k, op(B_b) is k×n. Blocks with k = 0 scale C_b by β. */
typedef struct tkb_gemm_desc {
  int64_t nblocks;
  const int64_t *m, *n, *k;
  const int64_t *offA, *offB, *offC;
  const int64_t *lda, *ldb, *ldc;
  const int32_t *opA, *opB;      /* tkb_op per block */
  int64_t lenA, lenB, lenC;      /* elements in each data vector (bounds check) */
  int32_t dtype;                 /* tkb_dtype */
  int32_t precision;             /* tkb_precision */
  int32_t slices;                /* split precision: int8 slices per operand. 0 = auto: up to 7,
                                    chosen per block on the device, with an FP64 fallback for
                                    blocks and tiles the slices cannot serve to 1e-12; 3..7 =
                                    exactly that many for every block, unchecked */
} tkb_gemm_desc;

int tkb_gemm_plan_create(tkb_ctx *ctx, const tkb_gemm_desc *desc, tkb_plan **out);
/* The same plan with the work-decomposition knobs set by the caller (an autotuner): when the
 * output tiles alone would leave SMs idle, the K loops are cut into at most max_pieces pieces
 * (1..64; 1 = no split K) of at least min_piece_steps K steps (BK = 16 plain, 32 split).
 * tkb_gemm_plan_create uses max_pieces = 8, min_piece_steps = 4. (No reference counterpart.) */
typedef struct tkb_gemm_tuning {
  int32_t max_pieces;
  int32_t min_piece_steps;
} tkb_gemm_tuning;
int tkb_gemm_plan_create_tuned(tkb_ctx *ctx, const tkb_gemm_desc *desc, const tkb_gemm_tuning *tuning,
                               tkb_plan **out);
int tkb_gemm_plan_destroy(tkb_plan *plan);
/* flops (real, 2mnk per real block, 8mnk per complex block) and the slice count used */
int tkb_gemm_plan_info(const tkb_plan *plan, double *flops, int32_t *slices);
int tkb_grouped_gemm(tkb_ctx *ctx, const tkb_plan *plan, void *C, const void *A,
                     const void *B, tkb_scalar alpha, tkb_scalar beta);
/* Split precision: the slice count each block used in the plan's last tkb_grouped_gemm (with
 * slices = 0 in the descriptor, chosen on the device from the block's exponents and row norms;
 * 0 = the block ran in FP64, -1 = no products: k = 0, a skinny block or a plain-precision plan),
 * in out[0 .. nblocks-1], and in out[nblocks] the number of output tiles whose a-posteriori error
 * check sent them to FP64. n must be at least nblocks + 1. Waits for the context's stream. (No
 * reference counterpart: the reference's mul! runs every block in FP64.) */
int tkb_gemm_plan_slices(tkb_ctx *ctx, const tkb_plan *plan, int32_t *out, int64_t n);

/* ---- weighted block reductions ------------------------------------------------------ */
/* Segments s: elements x[off_s + i*stride_s], i < count_s, weighted by weight_s (dim(c)).
 * NORM2: Σ_s w_s Σ_i |x|² ;  INNER: Σ_s w_s Σ_i conj(x)·y ;  TRACE: Σ_s w_s Σ_i x.
 * The result (re, im) is written to host memory after the stream completes. */
int tkb_rplan_create(tkb_ctx *ctx, int64_t nseg, const int64_t *off, const int64_t *count,
                     const int64_t *stride, const double *weight, int64_t len,
                     tkb_rplan **out);
int tkb_rplan_destroy(tkb_rplan *plan);
int tkb_reduce(tkb_ctx *ctx, const tkb_rplan *plan, int kind, int dtype, const void *x,
               const void *y, double *host_out);
/* same reduction, result left in device memory (2 doubles) without synchronising */
int tkb_reduce_async(tkb_ctx *ctx, const tkb_rplan *plan, int kind, int dtype,
                     const void *x, const void *y, double *dev_out);

/* Allocation-free variant of tkb_reduce. It has no counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc at all — code whose device memory is owned
 * entirely by another allocator (a Julia CUDA.jl memory pool, a framework that has reserved
 * the whole device) or code running where a device allocation may block or fail (a
 * finalizer, an out-of-memory recovery path). It needs no context, plan or workspace and
 * calls no allocating routine: its scratch (segment table, per-block partial sums, result;
 * about 57 KiB) is a static device array that every GPU loading the library holds until the
 * process exits. The caller passes the data vectors and host segment arrays (same meaning
 * as tkb_rplan_create) and receives (re, im) in host_out after the stream has completed.
 * Limits: at most 1024 segments (TKB_ERR_SIZE beyond that). The first call on a device
 * looks up the array's device address for that device and, with CUDA's lazy module
 * loading, loads the library's kernels onto the device, which can itself need device
 * memory: make it once per device at start-up (any valid call that reduces at least one
 * element), not first from an out-of-memory recovery path. Host-side staging uses a few KiB of the caller's stack. All
 * calls share the array, so calls that overlap on the GPU (other streams, other host threads)
 * race and must be serialised by the caller. */
int tkb_reduce_noalloc(int device, void *stream, int kind, int dtype, const void *x,
                       const void *y, int64_t len, int64_t nseg, const int64_t *off,
                       const int64_t *count, const int64_t *stride, const double *weight,
                       double *host_out);

/* ---- CUDA graph capture of a sequence of calls on the context stream ---------------- */
int tkb_graph_begin(tkb_ctx *ctx);
int tkb_graph_end(tkb_ctx *ctx, tkb_graph **out);
int tkb_graph_launch(tkb_ctx *ctx, const tkb_graph *graph);
int tkb_graph_destroy(tkb_graph *graph);

#ifdef __cplusplus
}
#endif
#endif /* TKB200_H */
