// Weighted block reductions for norm / inner / tr (src/tensors/linalg.jl:257-282, 319-327;
// src/tensors/vectorinterface.jl:114-130): Σ_c dim(c)·f(block_c), accumulated in FP64.
// Two deterministic passes: per-CTA partial sums over contiguous ranges of the segment
// element space, then one CTA sums the partials in a fixed order.
#include <algorithm>
#include <mutex>
#include <string>

#include "tkb_internal.h"

namespace {

constexpr int RT = 256;

__device__ __forceinline__ double2 term(int kind, const double *x, const double *y, int64_t i) {
  if (kind == TKB_NORM2) { const double v = x[i]; return make_double2(v * v, 0.0); }
  if (kind == TKB_INNER) return make_double2(x[i] * y[i], 0.0);
  return make_double2(x[i], 0.0);
}
__device__ __forceinline__ double2 term(int kind, const double2 *x, const double2 *y, int64_t i) {
  const double2 a = x[i];
  if (kind == TKB_NORM2) return make_double2(a.x * a.x + a.y * a.y, 0.0);
  if (kind == TKB_INNER) {
    const double2 b = y[i];
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);  // conj(a)·b
  }
  return a;
}

__device__ __forceinline__ double2 block_sum(double2 v) {
  __shared__ double2 red[RT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double2 r = make_double2(0.0, 0.0);
  if (threadIdx.x == 0)
    for (int w = 0; w < RT / 32; ++w) { r.x += red[w].x; r.y += red[w].y; }
  __syncthreads();
  return r;
}

template <typename T>
__global__ void __launch_bounds__(RT)
    reduce_partial_kernel(const RSeg *__restrict__ segs, const int64_t *__restrict__ seg_begin,
                          int64_t nseg, int64_t total, int kind, const T *__restrict__ x,
                          const T *__restrict__ y, double2 *__restrict__ partial) {
  const int64_t per = (total + gridDim.x - 1) / gridDim.x;
  const int64_t cb = (int64_t)blockIdx.x * per;
  const int64_t ce = min(total, cb + per);
  double2 acc = make_double2(0.0, 0.0);
  if (cb < ce) {
    int64_t gi = cb + threadIdx.x;
    // first segment containing gi
    int64_t lo = 0, hi = nseg - 1;
    const int64_t key = min(gi, total - 1);
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (seg_begin[mid] <= key) lo = mid; else hi = mid - 1;
    }
    int64_t s = lo;
    for (; gi < ce; gi += RT) {
      while (gi >= seg_begin[s + 1]) ++s;
      const RSeg sg = segs[s];
      const double2 v = term(kind, x, y, sg.off + (gi - seg_begin[s]) * sg.stride);
      acc.x = fma(sg.weight, v.x, acc.x);
      acc.y = fma(sg.weight, v.y, acc.y);
    }
  }
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void __launch_bounds__(RT) reduce_final_kernel(const double2 *__restrict__ partial,
                                                          int n, double *__restrict__ out) {
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < n; i += RT) { acc.x += partial[i].x; acc.y += partial[i].y; }
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) { out[0] = r.x; out[1] = r.y; }
}

}  // namespace

// ---- allocation-free variant ------------------------------------------------------------
// Scratch for tkb_reduce_noalloc: segment table, prefix sums, per-CTA partials and the
// result, in one file-scope device array that every GPU loading the library holds until
// the process exits. Host code only sees a stand-in for this symbol; its device address
// comes from cudaGetSymbolAddress, taken once per device.
namespace {
constexpr int64_t kNoAllocMaxSeg = 1024;
constexpr int kNoAllocMaxCta = 1024;
constexpr size_t kNoAllocSegBytes = kNoAllocMaxSeg * sizeof(RSeg);                 // 32 KiB
constexpr size_t kNoAllocBeginOff = kNoAllocSegBytes;
constexpr size_t kNoAllocPartialOff = (kNoAllocBeginOff + (kNoAllocMaxSeg + 1) * 8 + 255) / 256 * 256;
constexpr size_t kNoAllocResultOff = kNoAllocPartialOff + kNoAllocMaxCta * sizeof(double2);
constexpr size_t kNoAllocBytes = kNoAllocResultOff + 256;                          // ~57 KiB
}  // namespace

static __device__ __align__(256) unsigned char tkb_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {nullptr};
}  // namespace

extern "C" int tkb_reduce_noalloc(int device, void *stream, int kind, int dtype, const void *x,
                                  const void *y, int64_t len, int64_t nseg, const int64_t *off,
                                  const int64_t *count, const int64_t *stride, const double *weight,
                                  double *host_out) {
  if (kind < TKB_NORM2 || kind > TKB_TRACE) return tkb_set_error(nullptr, TKB_ERR_ARG, "unknown reduction");
  if (dtype != TKB_F64 && dtype != TKB_C128) return tkb_set_error(nullptr, TKB_ERR_ARG, "unknown dtype");
  if (!host_out) return tkb_set_error(nullptr, TKB_ERR_ARG, "null output");
  if (device < 0 || device >= 64) return tkb_set_error(nullptr, TKB_ERR_ARG, "device out of range");
  if (nseg < 0 || nseg > kNoAllocMaxSeg)
    return tkb_set_error(nullptr, TKB_ERR_SIZE,
                         "tkb_reduce_noalloc supports at most 1024 segments (got " +
                             std::to_string(nseg) + "); use tkb_reduce for larger tensors");
  if (nseg > 0 && (!off || !count || !stride || !weight))
    return tkb_set_error(nullptr, TKB_ERR_ARG, "null segment array");
  // validation (overflow-safe: count − 1 is compared with the room left after off)
  int64_t total = 0;
  for (int64_t s = 0; s < nseg; ++s) {
    if (count[s] < 0 || off[s] < 0 || stride[s] < 0)
      return tkb_set_error(nullptr, TKB_ERR_ARG, "invalid segment");
    if (count[s] > 0 && !tkb_segment_in_bounds(off[s], count[s], stride[s], len))
      return tkb_set_error(nullptr, TKB_ERR_SIZE, "segment outside the data vector");
    total += count[s];
  }
  if (total > 0 && (!x || (kind == TKB_INNER && !y)))
    return tkb_set_error(nullptr, TKB_ERR_ARG, "null data");

  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return tkb_set_error(nullptr, TKB_ERR_CUDA, cudaGetErrorString(e));
  unsigned char *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, tkb_noalloc_scratch);
      if (e != cudaSuccess) {
        cudaSetDevice(prev);
        return tkb_set_error(nullptr, TKB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
      g_noalloc_ptr[device] = p;
    }
    base = static_cast<unsigned char *>(g_noalloc_ptr[device]);
  }
  cudaStream_t st = (cudaStream_t)stream;
  RSeg *dsegs = reinterpret_cast<RSeg *>(base);
  int64_t *dbegin = reinterpret_cast<int64_t *>(base + kNoAllocBeginOff);
  double2 *dpart = reinterpret_cast<double2 *>(base + kNoAllocPartialOff);
  double *dres = reinterpret_cast<double *>(base + kNoAllocResultOff);
  e = cudaSuccess;
  if (total == 0) {
    host_out[0] = 0.0;
    host_out[1] = 0.0;
  } else {
    // The segment table and its prefix sums go up in chunks staged in small stack buffers
    // (a few KiB: callers such as finalizers may run on small stacks). The sources are pageable
    // host memory, so each copy has read its buffer when cudaMemcpyAsync returns and the buffer
    // can be refilled.
    constexpr int64_t kChunk = 64;
    RSeg segs[kChunk];
    int64_t begin[kChunk + 1];
    int64_t run = 0;
    for (int64_t s0 = 0; s0 < nseg && e == cudaSuccess; s0 += kChunk) {
      const int64_t n = std::min<int64_t>(kChunk, nseg - s0);
      for (int64_t q = 0; q < n; ++q) {
        const int64_t s = s0 + q;
        segs[q] = {off[s], count[s], stride[s], weight[s]};
        begin[q] = run;
        run += count[s];
      }
      begin[n] = run;
      e = cudaMemcpyAsync(dsegs + s0, segs, n * sizeof(RSeg), cudaMemcpyHostToDevice, st);
      // the prefix sums overlap by one entry between chunks (the same value is written twice)
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(dbegin + s0, begin, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
    }
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((total + 4095) / 4096, kNoAllocMaxCta));
    if (e == cudaSuccess) {
      if (dtype == TKB_F64)
        reduce_partial_kernel<double><<<nb, RT, 0, st>>>(dsegs, dbegin, nseg, total, kind,
                                                         (const double *)x, (const double *)y, dpart);
      else
        reduce_partial_kernel<double2><<<nb, RT, 0, st>>>(dsegs, dbegin, nseg, total, kind,
                                                          (const double2 *)x, (const double2 *)y, dpart);
      reduce_final_kernel<<<1, RT, 0, st>>>(dpart, nb, dres);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  cudaSetDevice(prev);
  if (e != cudaSuccess) return tkb_set_error(nullptr, TKB_ERR_CUDA, cudaGetErrorString(e));
  return TKB_OK;
}

int tkb_reduce_launch(tkb_ctx *ctx, const tkb_rplan *p, int kind, int dtype, const void *x,
                      const void *y, double *dev_out) {
  const int nb = p->nblocks_launch;
  // workspace layout: [partials (nb double2)]
  const size_t need = (size_t)nb * sizeof(double2);
  if (ctx->ws_bytes < need) return tkb_set_error(ctx, TKB_ERR_ARG, "workspace too small for reduction");
  double2 *partial = reinterpret_cast<double2 *>(ctx->ws);
  if (p->total == 0) {
    TKB_CUDA_TRY(ctx, cudaMemsetAsync(dev_out, 0, 2 * sizeof(double), ctx->stream));
    return TKB_OK;
  }
  if (dtype == TKB_F64)
    reduce_partial_kernel<double><<<nb, RT, 0, ctx->stream>>>(p->segs, p->seg_begin, p->nseg, p->total,
                                                             kind, (const double *)x, (const double *)y, partial);
  else
    reduce_partial_kernel<double2><<<nb, RT, 0, ctx->stream>>>(p->segs, p->seg_begin, p->nseg, p->total,
                                                              kind, (const double2 *)x, (const double2 *)y, partial);
  reduce_final_kernel<<<1, RT, 0, ctx->stream>>>(partial, nb, dev_out);
  ctx->launches += 2;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}
