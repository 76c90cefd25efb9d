// Partial-trace transform: every destination sub-block of a trace_permute! in one launch.
//
// Semantics (TensorKit _trace_permute!, src/tensors/tensoroperations.jl:246-296, bosonic):
//   dst_g = β·dst_g + α·Σ_e coeff_e · tensortrace(src_e, p, q)      for every group g
// where the entries e of group g are the source sub-blocks whose permuted tree pairs split
// into destination pair g. The host flattens the recoupling (permute of the fusion blocks to
// ((p₁, q₁), (p₂, q₂)), split, dim ratio) into coefficients; a traced leg pair becomes one
// summation index with stride stride(q₁) + stride(q₂).
//
// Work decomposition: one thread per destination element; CTAs take tasks of kTrThreads
// consecutive elements of one group (the destination's first dim is its fastest, so stores
// coalesce). Every element reads its entries' diagonals directly; traces are small side
// operations of a network (environment updates), not a bandwidth-critical path.
#include <algorithm>
#include <cstring>

#include "tkb_internal.h"

namespace {

constexpr int kTrThreads = 256;

struct CDbl {
  double x, y;
};

__device__ __forceinline__ double ld_src(const double *p, bool) { return __ldg(p); }
__device__ __forceinline__ double2 ld_src(const double2 *p, bool conj) {
  double2 v = __ldg(p);
  if (conj) v.y = -v.y;
  return v;
}
__device__ __forceinline__ double zero_v(double) { return 0.0; }
__device__ __forceinline__ double2 zero_v(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double add_v(double a, double b) { return a + b; }
__device__ __forceinline__ double2 add_v(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double axpy_v(double u, double v, double acc) { return fma(u, v, acc); }
__device__ __forceinline__ double2 axpy_v(double u, double2 v, double2 acc) {
  return make_double2(fma(u, v.x, acc.x), fma(u, v.y, acc.y));
}
__device__ __forceinline__ double finish_v(double v, CDbl a, CDbl b, const double *d, bool bz) {
  double r = a.x * v;
  if (!bz) r = fma(b.x, *d, r);
  return r;
}
__device__ __forceinline__ double2 finish_v(double2 v, CDbl a, CDbl b, const double2 *d, bool bz) {
  double2 r = make_double2(a.x * v.x - a.y * v.y, a.x * v.y + a.y * v.x);
  if (!bz) {
    const double2 o = *d;
    r.x = fma(b.x, o.x, fma(-b.y, o.y, r.x));
    r.y = fma(b.x, o.y, fma(b.y, o.x, r.y));
  }
  return r;
}

template <typename T, bool CONJ>
__global__ void __launch_bounds__(kTrThreads)
    trace_kernel(const TrGroup *__restrict__ groups, const TrEntry *__restrict__ entries,
                 const int32_t *__restrict__ task_group, int64_t ntasks, int nfree, int ntrace,
                 T *__restrict__ dst, const T *__restrict__ src, CDbl alpha, CDbl beta, int beta_zero) {
  const bool bz = beta_zero != 0;
  for (int64_t task = blockIdx.x; task < ntasks; task += gridDim.x) {
    const TrGroup &G = groups[task_group[task]];
    const int64_t e = (task - G.task_begin) * kTrThreads + threadIdx.x;
    if (e >= G.nelem) continue;
    // free multi-index (first dim fastest)
    int32_t x[TKB_MAX_IND];
    int64_t r = e, doff = G.dst_off;
#pragma unroll
    for (int k = 0; k < TKB_MAX_IND; ++k) {
      if (k < nfree) {
        x[k] = (int32_t)(r % G.size[k]);
        r /= G.size[k];
        doff += (int64_t)x[k] * G.dstr[k];
      } else {
        x[k] = 0;
      }
    }
    T acc = zero_v(T{});
    for (int64_t ei = G.e_begin; ei < G.e_end; ++ei) {
      const TrEntry &E = entries[ei];
      int64_t base = E.src_off;
#pragma unroll
      for (int k = 0; k < TKB_MAX_IND; ++k)
        if (k < nfree) base += (int64_t)x[k] * E.sstr[k];
      T s = zero_v(T{});
      for (int64_t t = 0; t < E.ntr_total; ++t) {
        int64_t rt = t, off = base;
#pragma unroll
        for (int l = 0; l < TKB_MAX_IND; ++l) {
          if (l < ntrace) {
            off += (rt % E.tsize[l]) * E.tstr[l];
            rt /= E.tsize[l];
          }
        }
        s = add_v(s, ld_src(src + off, CONJ));
      }
      acc = axpy_v(E.coeff, s, acc);
    }
    T *dp = dst + doff;
    *dp = finish_v(acc, alpha, beta, dp, bz);
  }
}

}  // namespace

extern "C" int tkb_trace_table_create(tkb_ctx *ctx, const tkb_trace_desc *d, tkb_trace_table **out) {
  if (!ctx || !d || !out) return TKB_ERR_ARG;
  *out = nullptr;
  const int nf = d->nfree, nt = d->ntrace;
  if (nf < 0 || nf > TKB_MAX_IND || nt < 1 || nt > TKB_MAX_IND)
    return tkb_set_error(ctx, TKB_ERR_ARG, "nfree/ntrace out of range");
  const int64_t G = d->ngroups;
  if (G < 0) return tkb_set_error(ctx, TKB_ERR_ARG, "negative ngroups");
  if (G > 0 && (!d->group_entry_ptr || !d->dst_offsets || (nf > 0 && (!d->sizes || !d->dst_strides))))
    return tkb_set_error(ctx, TKB_ERR_ARG, "null group array");
  const int64_t NE = G > 0 ? d->group_entry_ptr[G] : 0;
  if (NE > 0 && (!d->src_offsets || !d->coeffs || !d->trace_sizes || !d->trace_strides ||
                 (nf > 0 && !d->src_strides)))
    return tkb_set_error(ctx, TKB_ERR_ARG, "null entry array");
  std::vector<TrGroup> hg(G);
  std::vector<TrEntry> he(NE);
  std::vector<int32_t> htask;
  int64_t ntasks = 0;
  for (int64_t g = 0; g < G; ++g) {
    TrGroup &tg = hg[g];
    std::memset(&tg, 0, sizeof(tg));
    const int64_t e0 = d->group_entry_ptr[g], e1 = d->group_entry_ptr[g + 1];
    if (e0 < 0 || e1 < e0 || e1 > NE) return tkb_set_error(ctx, TKB_ERR_ARG, "inconsistent entry pointers");
    tg.e_begin = e0;
    tg.e_end = e1;
    tg.dst_off = d->dst_offsets[g];
    int64_t hi = tg.dst_off, vol = 1;
    if (hi < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative destination offset");
    for (int k = 0; k < nf; ++k) {
      const int64_t sz = d->sizes[g * nf + k], st = d->dst_strides[g * nf + k];
      if (sz <= 0 || sz > INT32_MAX) return tkb_set_error(ctx, TKB_ERR_SIZE, "bad free size");
      if (st < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative destination stride");
      tg.size[k] = (int32_t)sz;
      tg.dstr[k] = st;
      hi += (sz - 1) * st;
      vol *= sz;
    }
    if (hi >= d->dst_len)
      return tkb_set_error(ctx, TKB_ERR_SIZE, "destination sub-block exceeds its data vector");
    tg.nelem = vol;
    tg.task_begin = ntasks;
    const int64_t nt_g = (vol + kTrThreads - 1) / kTrThreads;
    htask.insert(htask.end(), (size_t)nt_g, (int32_t)g);
    ntasks += nt_g;
    for (int64_t e = e0; e < e1; ++e) {
      TrEntry &te = he[e];
      std::memset(&te, 0, sizeof(te));
      te.src_off = d->src_offsets[e];
      te.coeff = d->coeffs[e];
      int64_t shi = te.src_off, ntot = 1;
      if (shi < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative source offset");
      for (int k = 0; k < nf; ++k) {
        const int64_t st = d->src_strides[e * nf + k];
        if (st < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative source stride");
        te.sstr[k] = st;
        shi += (tg.size[k] - 1) * st;
      }
      for (int l = 0; l < nt; ++l) {
        const int64_t sz = d->trace_sizes[e * nt + l], st = d->trace_strides[e * nt + l];
        if (sz <= 0 || sz > INT32_MAX || st < 0)
          return tkb_set_error(ctx, TKB_ERR_SIZE, "bad traced size or stride");
        te.tsize[l] = (int32_t)sz;
        te.tstr[l] = st;
        shi += (sz - 1) * st;
        ntot *= sz;
      }
      te.ntr_total = ntot;
      if (shi >= d->src_len)
        return tkb_set_error(ctx, TKB_ERR_SIZE, "source sub-block exceeds its data vector");
    }
  }
  tkb_trace_table *t = new tkb_trace_table();
  t->owner = ctx;
  t->nfree = nf;
  t->ntrace = nt;
  t->ngroups = G;
  t->ntasks = ntasks;
  t->src_len = d->src_len;
  t->dst_len = d->dst_len;
  auto up = [&](void **dptr, const void *h, size_t bytes) -> cudaError_t {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(dptr, bytes);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dptr, h, bytes, cudaMemcpyHostToDevice);
  };
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = up((void **)&t->groups, hg.data(), hg.size() * sizeof(TrGroup));
  if (e == cudaSuccess) e = up((void **)&t->entries, he.data(), he.size() * sizeof(TrEntry));
  if (e == cudaSuccess) e = up((void **)&t->task_group, htask.data(), htask.size() * 4);
  if (e != cudaSuccess) {
    tkb_trace_table_destroy(t);
    return tkb_set_error(ctx, e == cudaErrorMemoryAllocation ? TKB_ERR_OOM : TKB_ERR_CUDA,
                         std::string("trace table upload: ") + cudaGetErrorString(e));
  }
  *out = t;
  return TKB_OK;
}

extern "C" int tkb_trace_table_destroy(tkb_trace_table *t) {
  if (!t) return TKB_OK;
  cudaFree(t->groups);
  cudaFree(t->entries);
  cudaFree(t->task_group);
  delete t;
  return TKB_OK;
}

extern "C" int tkb_tracetransform(tkb_ctx *ctx, const tkb_trace_table *t, int dtype, void *dst,
                                  const void *src, tkb_scalar alpha, tkb_scalar beta, int conj) {
  if (!ctx || !t) return TKB_ERR_ARG;
  if (t->owner != ctx) return tkb_set_error(ctx, TKB_ERR_ARG, "trace table belongs to another context");
  if (t->ntasks == 0) return TKB_OK;
  if (!dst || !src) return tkb_set_error(ctx, TKB_ERR_ARG, "null data pointer");
  const int grid = (int)std::min<int64_t>(t->ntasks, (int64_t)ctx->num_sms * 8);
  const CDbl a{alpha.re, alpha.im}, b{beta.re, beta.im};
  const int bz = (beta.re == 0.0 && beta.im == 0.0) ? 1 : 0;
  if (dtype == TKB_F64) {
    if (alpha.im != 0.0 || beta.im != 0.0)
      return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
    trace_kernel<double, false><<<grid, kTrThreads, 0, ctx->stream>>>(
        t->groups, t->entries, t->task_group, t->ntasks, t->nfree, t->ntrace, (double *)dst,
        (const double *)src, a, b, bz);
  } else if (dtype == TKB_C128) {
    auto k = conj ? trace_kernel<double2, true> : trace_kernel<double2, false>;
    k<<<grid, kTrThreads, 0, ctx->stream>>>(t->groups, t->entries, t->task_group, t->ntasks, t->nfree,
                                           t->ntrace, (double2 *)dst, (const double2 *)src, a, b, bz);
  } else {
    return tkb_set_error(ctx, TKB_ERR_ARG, "unknown dtype");
  }
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}
