// Weighted block reductions for norm / inner / tr (src/tensors/linalg.jl:257-282, 319-327;
// src/tensors/vectorinterface.jl:114-130): Σ_c dim(c)·f(block_c), accumulated in FP64.
// Two deterministic passes: per-CTA partial sums over contiguous ranges of the segment
// element space, then one CTA sums the partials in a fixed order.
#include <algorithm>

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
