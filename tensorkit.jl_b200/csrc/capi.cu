// C-ABI entry points of libtkb200: contexts, plans, dispatch and CUDA-graph capture.
// Every entry validates its arguments on the host (handles, sizes, every address a launch
// can touch) before anything is launched, and reports failures as status codes plus a
// message retrievable with tkb_last_error.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "tkb_internal.h"

namespace {
thread_local std::string g_err;
}

int tkb_set_error(tkb_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  g_err = msg;
  return code;
}

int tkb_ensure_workspace(tkb_ctx *ctx, size_t bytes) {
  if (bytes <= ctx->ws_bytes) return TKB_OK;
  if (ctx->in_capture)
    return tkb_set_error(ctx, TKB_ERR_ARG, "workspace growth requested during graph capture");
  // the stream may still use the old workspace
  TKB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->ws);
  ctx->ws = nullptr;
  ctx->ws_bytes = 0;
  const size_t nb = (bytes + 255) / 256 * 256;
  cudaError_t e = cudaMalloc(&ctx->ws, nb);
  if (e != cudaSuccess) return tkb_set_error(ctx, TKB_ERR_OOM, "workspace allocation failed");
  ctx->ws_bytes = nb;
  return TKB_OK;
}

extern "C" {

int tkb_version(void) { return 200; }

const char *tkb_last_error(const tkb_ctx *ctx) {
  if (ctx) return ctx->err.c_str();
  return g_err.c_str();
}

int tkb_ctx_create(int device, void *stream, size_t workspace_bytes, tkb_ctx **out) {
  if (!out) return tkb_set_error(nullptr, TKB_ERR_ARG, "null output handle");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return tkb_set_error(nullptr, TKB_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= ndev) return tkb_set_error(nullptr, TKB_ERR_ARG, "device out of range");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return tkb_set_error(nullptr, TKB_ERR_CUDA, cudaGetErrorString(e));
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return tkb_set_error(nullptr, TKB_ERR_CUDA, cudaGetErrorString(e));
  if (prop.major != 10)
    return tkb_set_error(nullptr, TKB_ERR_UNSUPPORTED, "libtkb200 is built for sm_100a (B200)");
  tkb_ctx *ctx = new tkb_ctx();
  ctx->device = device;
  ctx->stream = (cudaStream_t)stream;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->smem_optin = prop.sharedMemPerBlockOptin;
  e = cudaMalloc((void **)&ctx->counters, 64 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(ctx->counters, 0, 64 * sizeof(int));
  if (e != cudaSuccess) {
    delete ctx;
    return tkb_set_error(nullptr, TKB_ERR_OOM, "counter allocation failed");
  }
  const size_t ws = std::max<size_t>(workspace_bytes, 1 << 20);
  if (tkb_ensure_workspace(ctx, ws) != TKB_OK) {
    cudaFree(ctx->counters);
    delete ctx;
    return tkb_set_error(nullptr, TKB_ERR_OOM, "workspace allocation failed");
  }
  *out = ctx;
  return TKB_OK;
}

int tkb_ctx_destroy(tkb_ctx *ctx) {
  if (!ctx) return TKB_OK;
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->ws);
  cudaFree(ctx->counters);
  delete ctx;
  return TKB_OK;
}

int tkb_ctx_set_stream(tkb_ctx *ctx, void *stream) {
  if (!ctx) return tkb_set_error(nullptr, TKB_ERR_ARG, "null context");
  if (ctx->in_capture) return tkb_set_error(ctx, TKB_ERR_ARG, "cannot change stream during capture");
  ctx->stream = (cudaStream_t)stream;
  return TKB_OK;
}

// ctx->counters[kErrSlot]: codes of bounded device waits that gave up (kernels set it with
// atomicExch, the host reads and clears it at synchronisation)
constexpr int kErrSlot = 8, kNeverSetSlot = 10;

int tkb_ctx_synchronize(tkb_ctx *ctx) {
  if (!ctx) return tkb_set_error(nullptr, TKB_ERR_ARG, "null context");
  TKB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  int code = 0;
  TKB_CUDA_TRY(ctx, cudaMemcpyAsync(&code, ctx->counters + kErrSlot, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TKB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (code != 0) {
    TKB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->counters + kErrSlot, 0, sizeof(int), ctx->stream));
    TKB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    static const char *what[] = {"", "split GEMM: a shared-memory ring stage did not arrive",
                                 "split GEMM: the tensor-core products did not complete",
                                 "split GEMM: the split-K pieces of a tile did not all arrive",
                                 "bounded-wait self-test: the flag was never set"};
    return tkb_set_error(ctx, TKB_ERR_TIMEOUT,
                         std::string("bounded device wait gave up: ") + (code >= 1 && code <= 4 ? what[code] : "unknown"));
  }
  return TKB_OK;
}

namespace {
// one thread waits (bounded by %globaltimer) on a flag that nothing sets, then records code 4
__global__ void bounded_wait_selftest_kernel(const int *flag, int *err, long long timeout_ns) {
  if (threadIdx.x != 0) return;
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t0));
  while (true) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(flag) : "memory");
    if (v != 0) return;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    if ((long long)(t - t0) > timeout_ns) {
      atomicExch(err, 4);
      return;
    }
    __nanosleep(1000);
  }
}
}  // namespace

int tkb_selftest_bounded_wait(tkb_ctx *ctx, int64_t timeout_us) {
  if (!ctx) return tkb_set_error(nullptr, TKB_ERR_ARG, "null context");
  if (timeout_us < 1 || timeout_us > 1000000) return tkb_set_error(ctx, TKB_ERR_ARG, "timeout_us must be in 1 .. 1000000");
  bounded_wait_selftest_kernel<<<1, 32, 0, ctx->stream>>>(ctx->counters + kNeverSetSlot, ctx->counters + kErrSlot,
                                                          (long long)timeout_us * 1000);
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

int tkb_ctx_launch_count(const tkb_ctx *ctx, int64_t *count) {
  if (!ctx || !count) return TKB_ERR_ARG;
  *count = ctx->launches;
  return TKB_OK;
}

int tkb_treetransform(tkb_ctx *ctx, const tkb_table *t, int dtype, void *dst, const void *src,
                      tkb_scalar alpha, tkb_scalar beta, int conj_src) {
  if (!ctx || !t) return tkb_set_error(ctx, TKB_ERR_ARG, "null context or table");
  if (t->owner != ctx) return tkb_set_error(ctx, TKB_ERR_ARG, "table belongs to another context");
  if (t->ntasks > 0 && (!dst || !src)) return tkb_set_error(ctx, TKB_ERR_ARG, "null data pointer");
  if (dtype != TKB_F64 && dtype != TKB_C128) return tkb_set_error(ctx, TKB_ERR_ARG, "unknown dtype");
  return tkb_transform_launch(ctx, t, dtype, dst, src, alpha, beta, conj_src);
}

// ---- grouped gemm plans ---------------------------------------------------------------
static bool in_bounds(int64_t off, int64_t rows, int64_t cols, int64_t ld, int64_t len) {
  if (rows == 0 || cols == 0) return true;
  if (off < 0 || ld < rows) return false;
  return off + (rows - 1) + (cols - 1) * ld < len;
}

static int plan_create(tkb_ctx *ctx, const tkb_gemm_desc *d, const tkb_gemm_tuning *tn, tkb_plan **out);

int tkb_gemm_plan_create(tkb_ctx *ctx, const tkb_gemm_desc *d, tkb_plan **out) {
  return plan_create(ctx, d, nullptr, out);
}

int tkb_gemm_plan_create_tuned(tkb_ctx *ctx, const tkb_gemm_desc *d, const tkb_gemm_tuning *t, tkb_plan **out) {
  if (!t) return tkb_set_error(ctx, TKB_ERR_ARG, "null tuning");
  if (t->max_pieces < 1 || t->max_pieces > 64 || t->min_piece_steps < 1)
    return tkb_set_error(ctx, TKB_ERR_ARG, "tuning: max_pieces must be in 1..64, min_piece_steps at least 1");
  return plan_create(ctx, d, t, out);
}

static int plan_create(tkb_ctx *ctx, const tkb_gemm_desc *d, const tkb_gemm_tuning *tn, tkb_plan **out) {
  if (!ctx || !d || !out) return tkb_set_error(ctx, TKB_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->dtype != TKB_F64 && d->dtype != TKB_C128) return tkb_set_error(ctx, TKB_ERR_ARG, "unknown dtype");
  if (d->precision != TKB_PLAIN && d->precision != TKB_SPLIT_INT8)
    return tkb_set_error(ctx, TKB_ERR_ARG, "unknown precision");
  const int64_t nb = d->nblocks;
  if (nb < 0) return tkb_set_error(ctx, TKB_ERR_ARG, "negative block count");
  if (nb > 0 && (!d->m || !d->n || !d->k || !d->offA || !d->offB || !d->offC || !d->lda ||
                 !d->ldb || !d->ldc || !d->opA || !d->opB))
    return tkb_set_error(ctx, TKB_ERR_ARG, "null descriptor array");
  tkb_plan *p = new tkb_plan();
  p->owner = ctx;
  p->dtype = d->dtype;
  p->precision = d->precision;
  p->slices = d->slices;
  p->nblocks = nb;
  if (tn) {
    p->max_pieces = tn->max_pieces;
    p->min_piece_steps = tn->min_piece_steps;
  }
  p->lenA = d->lenA;
  p->lenB = d->lenB;
  p->lenC = d->lenC;
  std::vector<GTile> tiles, sk;
  double flops = 0;
  for (int64_t i = 0; i < nb; ++i) {
    GBlock b;
    std::memset(&b, 0, sizeof(b));
    b.m = d->m[i]; b.n = d->n[i]; b.k = d->k[i];
    b.offA = d->offA[i]; b.offB = d->offB[i]; b.offC = d->offC[i];
    b.lda = d->lda[i]; b.ldb = d->ldb[i]; b.ldc = d->ldc[i];
    b.opA = d->opA[i]; b.opB = d->opB[i];
    if (b.m < 0 || b.n < 0 || b.k < 0 || b.opA < 0 || b.opA > 2 || b.opB < 0 || b.opB > 2) {
      delete p;
      return tkb_set_error(ctx, TKB_ERR_ARG, "invalid block descriptor");
    }
    const bool okA = b.k == 0 || (b.opA == TKB_OP_N ? in_bounds(b.offA, b.m, b.k, b.lda, d->lenA)
                                                     : in_bounds(b.offA, b.k, b.m, b.lda, d->lenA));
    const bool okB = b.k == 0 || (b.opB == TKB_OP_N ? in_bounds(b.offB, b.k, b.n, b.ldb, d->lenB)
                                                     : in_bounds(b.offB, b.n, b.k, b.ldb, d->lenB));
    const bool okC = in_bounds(b.offC, b.m, b.n, b.ldc, d->lenC);
    if (!okA || !okB || !okC) {
      delete p;
      return tkb_set_error(ctx, TKB_ERR_SIZE, "block " + std::to_string(i) + " addresses outside its data vector");
    }
    if (d->dtype == TKB_F64 && (b.opA == TKB_OP_C || b.opB == TKB_OP_C)) {
      // conjugation of real data is the identity
      if (b.opA == TKB_OP_C) b.opA = TKB_OP_T;
      if (b.opB == TKB_OP_C) b.opB = TKB_OP_T;
    }
    flops += (d->dtype == TKB_C128 ? 8.0 : 2.0) * (double)b.m * (double)b.n * (double)b.k;
    b.skinny = (b.n <= kSkinnyMax && b.k <= kSkinnyMax && b.m >= kSkinnyMinRows) ? 1 : 0;
    if (b.skinny && b.m > 0 && b.n > 0) p->sk_dim = std::max<int>(p->sk_dim, (int)std::max(b.n, b.k));
    p->hblocks.push_back(b);
    if (b.m > 0 && b.n > 0) {
      if (b.skinny) {
        for (int64_t m0 = 0; m0 < b.m; m0 += kSkinnyTaskRows)
          sk.push_back({(int32_t)i, (int32_t)m0, 0, b.k > 0 ? 0 : 1});
      } else {
        for (int64_t m0 = 0; m0 < b.m; m0 += 64)
          for (int64_t n0 = 0; n0 < b.n; n0 += 64)
            tiles.push_back({(int32_t)i, (int32_t)m0, (int32_t)n0, b.k > 0 ? 0 : 1});
      }
    }
  }
  p->nsk = (int64_t)sk.size();
  std::stable_sort(tiles.begin(), tiles.end(), [&](const GTile &x, const GTile &y) {
    return p->hblocks[x.block].k > p->hblocks[y.block].k;
  });
  p->flops = flops;
  p->ntiles = (int64_t)tiles.size();
  int rc = TKB_OK;
  if (d->precision == TKB_SPLIT_INT8) rc = tkb_gemm_split_prepare(ctx, p);
  else rc = tkb_gemm_plain_prepare(ctx, p, tiles);
  if (rc != TKB_OK) {
    tkb_gemm_plan_destroy(p);
    return rc;
  }
  cudaError_t e = cudaSuccess;
  if (!p->hblocks.empty()) {
    e = cudaMalloc((void **)&p->blocks, p->hblocks.size() * sizeof(GBlock));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->blocks, p->hblocks.data(), p->hblocks.size() * sizeof(GBlock), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !tiles.empty()) {
    e = cudaMalloc((void **)&p->tiles, tiles.size() * sizeof(GTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->tiles, tiles.data(), tiles.size() * sizeof(GTile), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !sk.empty()) {
    e = cudaMalloc((void **)&p->sktasks, sk.size() * sizeof(GTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->sktasks, sk.data(), sk.size() * sizeof(GTile), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    tkb_gemm_plan_destroy(p);
    return tkb_set_error(ctx, TKB_ERR_CUDA, std::string("plan upload: ") + cudaGetErrorString(e));
  }
  *out = p;
  return TKB_OK;
}

int tkb_gemm_plan_destroy(tkb_plan *p) {
  if (!p) return TKB_OK;
  cudaFree(p->blocks);
  cudaFree(p->tiles);
  cudaFree(p->sktasks);
  cudaFree(p->ptasks);
  cudaFree(p->bstat);
  cudaFree(p->bslices);
  cudaFree(p->kstiles);
  cudaFree(p->part);
  cudaFree(p->pcnt);
  cudaFree(p->stiles);
  cudaFree(p->sjobs);
  delete p;
  return TKB_OK;
}

int tkb_gemm_plan_info(const tkb_plan *p, double *flops, int32_t *slices) {
  if (!p) return TKB_ERR_ARG;
  if (flops) *flops = p->flops;
  if (slices) *slices = p->precision == TKB_SPLIT_INT8 ? p->slices : 0;
  return TKB_OK;
}

int tkb_gemm_plan_slices(tkb_ctx *ctx, const tkb_plan *p, int32_t *out, int64_t n) {
  if (!ctx || !p || !out) return tkb_set_error(ctx, TKB_ERR_ARG, "null argument");
  if (p->owner != ctx) return tkb_set_error(ctx, TKB_ERR_ARG, "plan belongs to another context");
  const int64_t nb = (int64_t)p->hblocks.size();
  if (n < nb + 1) return tkb_set_error(ctx, TKB_ERR_ARG, "output array shorter than nblocks + 1");
  if (!p->bslices) {
    for (int64_t i = 0; i < nb; ++i) out[i] = -1;
    out[nb] = 0;
    return TKB_OK;
  }
  TKB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  TKB_CUDA_TRY(ctx, cudaMemcpy(out, p->bslices, (size_t)(nb + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return TKB_OK;
}

int tkb_grouped_gemm(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B,
                     tkb_scalar alpha, tkb_scalar beta) {
  if (!ctx || !p) return tkb_set_error(ctx, TKB_ERR_ARG, "null context or plan");
  if (p->owner != ctx) return tkb_set_error(ctx, TKB_ERR_ARG, "plan belongs to another context");
  if (p->nblocks > 0 && (!C || (p->flops > 0 && (!A || !B))))
    return tkb_set_error(ctx, TKB_ERR_ARG, "null data pointer");
  const int rc = tkb_gemm_skinny_launch(ctx, p, C, A, B, alpha, beta);
  if (rc != TKB_OK) return rc;
  if (p->precision == TKB_SPLIT_INT8) return tkb_gemm_split_launch(ctx, p, C, A, B, alpha, beta);
  return tkb_gemm_launch(ctx, p, C, A, B, alpha, beta);
}

// ---- reductions ------------------------------------------------------------------------
int tkb_rplan_create(tkb_ctx *ctx, int64_t nseg, const int64_t *off, const int64_t *count,
                     const int64_t *stride, const double *weight, int64_t len, tkb_rplan **out) {
  if (!ctx || !out || nseg < 0) return tkb_set_error(ctx, TKB_ERR_ARG, "invalid argument");
  *out = nullptr;
  if (nseg > 0 && (!off || !count || !stride || !weight))
    return tkb_set_error(ctx, TKB_ERR_ARG, "null segment array");
  std::vector<RSeg> segs(nseg);
  std::vector<int64_t> begin(nseg + 1, 0);
  for (int64_t s = 0; s < nseg; ++s) {
    if (count[s] < 0 || off[s] < 0 || stride[s] < 0)
      return tkb_set_error(ctx, TKB_ERR_ARG, "invalid segment");
    if (count[s] > 0 && !tkb_segment_in_bounds(off[s], count[s], stride[s], len))
      return tkb_set_error(ctx, TKB_ERR_SIZE, "segment outside the data vector");
    segs[s] = {off[s], count[s], stride[s], weight[s]};
    begin[s + 1] = begin[s] + count[s];
  }
  tkb_rplan *p = new tkb_rplan();
  p->owner = ctx;
  p->nseg = nseg;
  p->total = begin[nseg];
  p->nblocks_launch = (int)std::max<int64_t>(1, std::min<int64_t>((p->total + 4095) / 4096, (int64_t)ctx->num_sms * 4));
  cudaError_t e = cudaSuccess;
  if (nseg > 0) {
    e = cudaMalloc((void **)&p->segs, nseg * sizeof(RSeg));
    if (e == cudaSuccess) e = cudaMemcpy(p->segs, segs.data(), nseg * sizeof(RSeg), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc((void **)&p->seg_begin, (nseg + 1) * 8);
  if (e == cudaSuccess) e = cudaMemcpy(p->seg_begin, begin.data(), (nseg + 1) * 8, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    tkb_rplan_destroy(p);
    return tkb_set_error(ctx, TKB_ERR_CUDA, std::string("rplan upload: ") + cudaGetErrorString(e));
  }
  const int rc = tkb_ensure_workspace(ctx, (size_t)p->nblocks_launch * 16);
  if (rc != TKB_OK) {
    tkb_rplan_destroy(p);
    return rc;
  }
  *out = p;
  return TKB_OK;
}

int tkb_rplan_destroy(tkb_rplan *p) {
  if (!p) return TKB_OK;
  cudaFree(p->segs);
  cudaFree(p->seg_begin);
  delete p;
  return TKB_OK;
}

int tkb_reduce_async(tkb_ctx *ctx, const tkb_rplan *p, int kind, int dtype, const void *x,
                     const void *y, double *dev_out) {
  if (!ctx || !p || !dev_out) return tkb_set_error(ctx, TKB_ERR_ARG, "null argument");
  if (p->owner != ctx) return tkb_set_error(ctx, TKB_ERR_ARG, "plan belongs to another context");
  if (kind < TKB_NORM2 || kind > TKB_TRACE) return tkb_set_error(ctx, TKB_ERR_ARG, "unknown reduction");
  if (dtype != TKB_F64 && dtype != TKB_C128) return tkb_set_error(ctx, TKB_ERR_ARG, "unknown dtype");
  if (p->total > 0 && (!x || (kind == TKB_INNER && !y))) return tkb_set_error(ctx, TKB_ERR_ARG, "null data");
  return tkb_reduce_launch(ctx, p, kind, dtype, x, y, dev_out);
}

int tkb_reduce(tkb_ctx *ctx, const tkb_rplan *p, int kind, int dtype, const void *x,
               const void *y, double *host_out) {
  if (!host_out) return tkb_set_error(ctx, TKB_ERR_ARG, "null output");
  if (!ctx) return tkb_set_error(nullptr, TKB_ERR_ARG, "null context");
  // the last 32 bytes of the counter block hold the device-side result
  double *dres = reinterpret_cast<double *>(ctx->counters + 32);
  int rc = tkb_reduce_async(ctx, p, kind, dtype, x, y, dres);
  if (rc != TKB_OK) return rc;
  TKB_CUDA_TRY(ctx, cudaMemcpyAsync(host_out, dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TKB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return TKB_OK;
}

// ---- graphs ----------------------------------------------------------------------------
struct tkb_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  tkb_ctx *owner = nullptr;
};

int tkb_graph_begin(tkb_ctx *ctx) {
  if (!ctx) return tkb_set_error(nullptr, TKB_ERR_ARG, "null context");
  if (ctx->stream == nullptr) return tkb_set_error(ctx, TKB_ERR_ARG, "graph capture needs a non-default stream");
  if (ctx->in_capture) return tkb_set_error(ctx, TKB_ERR_ARG, "capture already active");
  TKB_CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  ctx->in_capture = true;
  return TKB_OK;
}

int tkb_graph_end(tkb_ctx *ctx, tkb_graph **out) {
  if (!ctx || !out) return tkb_set_error(ctx, TKB_ERR_ARG, "null argument");
  if (!ctx->in_capture) return tkb_set_error(ctx, TKB_ERR_ARG, "no capture active");
  ctx->in_capture = false;
  cudaGraph_t g = nullptr;
  TKB_CUDA_TRY(ctx, cudaStreamEndCapture(ctx->stream, &g));
  tkb_graph *h = new tkb_graph();
  h->graph = g;
  h->owner = ctx;
  cudaError_t e = cudaGraphInstantiate(&h->exec, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    delete h;
    return tkb_set_error(ctx, TKB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  *out = h;
  return TKB_OK;
}

int tkb_graph_launch(tkb_ctx *ctx, const tkb_graph *g) {
  if (!ctx || !g) return tkb_set_error(ctx, TKB_ERR_ARG, "null argument");
  TKB_CUDA_TRY(ctx, cudaGraphLaunch(g->exec, ctx->stream));
  return TKB_OK;
}

int tkb_graph_destroy(tkb_graph *g) {
  if (!g) return TKB_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return TKB_OK;
}

}  // extern "C"
