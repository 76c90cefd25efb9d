// Tree transform: gather-permute-recouple-scale-scatter of all sub-blocks of one
// permute/braid in a single launch.
//
// Semantics (TensorKit add_transform_kernel!, src/tensors/indexmanipulations.jl:658-726):
//   for every group g (a fusion block, or one abelian tree pair):
//     dst_i = β·dst_i + α·Σ_j U_g[i,j] · permutedims(src_j, perm)      i < ndst_g, j < nsrc_g
// A group's sub-blocks share their sizes; only strides/offsets differ per tree.
//
// Work decomposition: every group is canonicalised on the host (size-1 dims removed,
// dims contiguous on both sides merged) and tiled over two dims (a, b):
//   copy mode      a is the fastest dim of both source and destination: loads and stores
//                  are coalesced along a, source tiles staged in shared memory only when
//                  the group recouples several trees;
//   transpose mode a is the destination's fastest dim, b the source's: the source tile is
//                  read coalesced along b into shared memory (row pitch tb+1 to avoid bank
//                  conflicts) and written coalesced along a.
// All remaining dims are "outer": one task = one (tile_a, tile_b, outer index) of a group.
// Tasks of all groups form one grid; groups arrive sorted by decreasing weight.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include <mutex>
#include <unordered_map>

#include "tkb_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kBatch = 8;  // elements per thread per load batch (loads in flight per thread)
constexpr int kBatchPairs = kBatch / 2;  // 16-byte pairs per thread per batch
constexpr int64_t kTileElemsMax = 2048;  // largest task (= kThreads * kBatch elements)
constexpr size_t kSmemBudget = 96 * 1024;
constexpr int kTaskWords = 2 + TKB_MAX_IND;  // per task: tile a, tile b, outer multi-index

struct CDbl {
  double x, y;
};

__device__ __forceinline__ double ld_val(const double *p, bool) { return __ldg(p); }
__device__ __forceinline__ double2 ld_val(const double2 *p, bool conj) {
  double2 v = __ldg(p);
  if (conj) v.y = -v.y;
  return v;
}
__device__ __forceinline__ double zero_val(double) { return 0.0; }
__device__ __forceinline__ double2 zero_val(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double axpy_r(double u, double v, double acc) { return fma(u, v, acc); }
__device__ __forceinline__ double2 axpy_r(double u, double2 v, double2 acc) {
  return make_double2(fma(u, v.x, acc.x), fma(u, v.y, acc.y));
}
// out = α·v + β·d   (β_zero: d not read)
__device__ __forceinline__ double finish(double v, double a, double b, const double *d,
                                         bool bz) {
  double r = a * v;
  if (!bz) r = fma(b, *d, r);
  return r;
}
__device__ __forceinline__ double2 finish(double2 v, double2 a, double2 b, const double2 *d,
                                          bool bz) {
  double2 r = make_double2(a.x * v.x - a.y * v.y, a.x * v.y + a.y * v.x);
  if (!bz) {
    double2 o = *d;
    r.x = fma(b.x, o.x, fma(-b.y, o.y, r.x));
    r.y = fma(b.x, o.y, fma(b.y, o.x, r.y));
  }
  return r;
}

template <typename T>
__device__ __forceinline__ T scalar_from(CDbl s);
template <>
__device__ __forceinline__ double scalar_from<double>(CDbl s) { return s.x; }
template <>
__device__ __forceinline__ double2 scalar_from<double2>(CDbl s) { return make_double2(s.x, s.y); }

template <typename T, bool CONJ>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 8 ? 3 : 2)
    treetransform_kernel(const TGroup *__restrict__ groups, const int32_t *__restrict__ task_group,
                         const int32_t *__restrict__ task_idx, int64_t ntasks,
                         const int64_t *__restrict__ sstr,
                         const int64_t *__restrict__ soff, const int64_t *__restrict__ dstr,
                         const int64_t *__restrict__ doff, const double *__restrict__ coeffs,
                         T *__restrict__ dst, const T *__restrict__ src, CDbl alpha_, CDbl beta_,
                         int beta_zero) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const T alpha = scalar_from<T>(alpha_);
  const T beta = scalar_from<T>(beta_);
  const bool bz = beta_zero != 0;
  pdl_wait();     // source and destination belong to earlier kernels of the stream too
  pdl_trigger();  // the next kernel may be scheduled; it waits for this grid before reading

  // Each CTA walks a contiguous range of tasks (tasks of one group are contiguous, so the
  // group metadata stays in L1); the task → group map was built on the host.
  const int64_t per = (ntasks + gridDim.x - 1) / gridDim.x;
  const int64_t t_begin = (int64_t)blockIdx.x * per;
  const int64_t t_end = min(ntasks, t_begin + per);
  for (int64_t task = t_begin; task < t_end; ++task) {
    const TGroup &G = groups[task_group[task]];
    // tile coordinates and outer multi-index of the task, decomposed on the host
    const int32_t *tix = task_idx + task * kTaskWords;
    const int64_t ita = tix[0], itb = tix[1];
    int64_t oidx[TKB_MAX_IND];
#pragma unroll
    for (int q = 0; q < TKB_MAX_IND; ++q) oidx[q] = q < G.nouter ? tix[2 + q] : 0;
    const int da = G.da, db = G.db;
    const int ta = G.ta, tb = G.tb;
    const int64_t a0 = ita * ta, b0 = itb * tb;
    const int64_t sa = G.size[da];
    const int64_t sb = db >= 0 ? G.size[db] : 1;
    const int na = (int)(sa - a0 < ta ? sa - a0 : ta);
    const int nb = (int)(sb - b0 < tb ? sb - b0 : tb);
    const int nel = na * nb;
    const int64_t nsrc = G.nsrc, ndst = G.ndst;

    auto src_base = [&](int64_t j) {
      const int64_t *st = sstr + (G.src_tree_begin + j) * TKB_MAX_IND;
      int64_t off = soff[G.src_tree_begin + j] + a0 * st[da] + (db >= 0 ? b0 * st[db] : 0);
#pragma unroll
      for (int q = 0; q < TKB_MAX_IND; ++q)
        if (q < G.nouter) off += oidx[q] * st[G.outer[q]];
      return off;
    };
    auto dst_base = [&](int64_t i) {
      const int64_t *st = dstr + (G.dst_tree_begin + i) * TKB_MAX_IND;
      int64_t off = doff[G.dst_tree_begin + i] + a0 * st[da] + (db >= 0 ? b0 * st[db] : 0);
#pragma unroll
      for (int q = 0; q < TKB_MAX_IND; ++q)
        if (q < G.nouter) off += oidx[q] * st[G.outer[q]];
      return off;
    };

    // Tile extents are powers of two: index decomposition by shifts and masks, elements
    // outside the (na, nb) corner are skipped. Every thread issues its loads of a batch of
    // kBatch elements before using any of them, so each thread keeps kBatch loads in flight.
    const int lta = __ffs(ta) - 1, ltb = __ffs(tb) - 1;
    const int tot = ta * tb;
    (void)nel;

    if (G.mode == 0 && nsrc == 1 && ndst == 1) {
      // direct copy: coalesced along a on both sides
      const int64_t *ss = sstr + G.src_tree_begin * TKB_MAX_IND;
      const int64_t *ds = dstr + G.dst_tree_begin * TKB_MAX_IND;
      const int64_t sA = ss[da], dA = ds[da];
      const int64_t sB = db >= 0 ? ss[db] : 0, dB = db >= 0 ? ds[db] : 0;
      const int64_t sb0 = src_base(0), db0 = dst_base(0);
      const double u = coeffs[G.coeff_begin];
      for (int e0 = 0; e0 < tot; e0 += kThreads * kBatch) {
        T v[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
          const int e = e0 + q * kThreads + threadIdx.x;
          const int ia = e & (ta - 1), ib = e >> lta;
          v[q] = (e < tot && ia < na && ib < nb) ? ld_val(src + sb0 + ia * sA + ib * sB, CONJ)
                                                : zero_val(T{});
        }
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
          const int e = e0 + q * kThreads + threadIdx.x;
          const int ia = e & (ta - 1), ib = e >> lta;
          if (e < tot && ia < na && ib < nb) {
            T *dp = dst + db0 + ia * dA + ib * dB;
            *dp = finish(axpy_r(u, v[q], zero_val(T{})), alpha, beta, dp, bz);
          }
        }
      }
      continue;
    }

    // staged path: all source tiles of the group into shared memory
    const int pitch = (G.mode == 1) ? (tb + 1) : 0;
    const int tile_elems = (G.mode == 1) ? ta * (tb + 1) : ta * tb;
    for (int64_t j = 0; j < nsrc; ++j) {
      const int64_t *ss = sstr + (G.src_tree_begin + j) * TKB_MAX_IND;
      const int64_t sA = ss[da], sB = db >= 0 ? ss[db] : 0;
      const int64_t base = src_base(j);
      T *tile = sm + j * tile_elems;
      for (int e0 = 0; e0 < tot; e0 += kThreads * kBatch) {
        T v[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
          const int e = e0 + q * kThreads + threadIdx.x;
          // transpose mode: b fastest (coalesced source reads); copy mode: a fastest
          const int ia = G.mode == 1 ? (e >> ltb) : (e & (ta - 1));
          const int ib = G.mode == 1 ? (e & (tb - 1)) : (e >> lta);
          v[q] = (e < tot && ia < na && ib < nb) ? ld_val(src + base + ia * sA + ib * sB, CONJ)
                                                : zero_val(T{});
        }
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
          const int e = e0 + q * kThreads + threadIdx.x;
          const int ia = G.mode == 1 ? (e >> ltb) : (e & (ta - 1));
          const int ib = G.mode == 1 ? (e & (tb - 1)) : (e >> lta);
          if (e < tot) tile[G.mode == 1 ? ia * pitch + ib : ib * ta + ia] = v[q];
        }
      }
    }
    __syncthreads();
    const double *U = coeffs + G.coeff_begin;
    for (int64_t i = 0; i < ndst; ++i) {
      const int64_t *ds = dstr + (G.dst_tree_begin + i) * TKB_MAX_IND;
      const int64_t dA = ds[da], dB = db >= 0 ? ds[db] : 0;
      const int64_t base = dst_base(i);
      const double *Ui = U + i * nsrc;
      for (int e0 = 0; e0 < tot; e0 += kThreads * kBatch) {
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
          const int e = e0 + q * kThreads + threadIdx.x;
          const int ia = e & (ta - 1), ib = e >> lta;  // a fastest: coalesced destination writes
          if (e < tot && ia < na && ib < nb) {
            const int sidx = (G.mode == 1) ? ia * pitch + ib : ib * ta + ia;
            T acc = zero_val(T{});
            for (int64_t j = 0; j < nsrc; ++j) acc = axpy_r(Ui[j], sm[j * tile_elems + sidx], acc);
            T *dp = dst + base + ia * dA + ib * dB;
            *dp = finish(acc, alpha, beta, dp, bz);
          }
        }
      }
    }
    __syncthreads();
  }
}

// ---- pipelined kernel for tables of single-tree groups (nsrc = ndst = 1) -----------------
// Abelian transformers and fusion blocks with one tree pair are pure strided copies with one
// coefficient. A persistent CTA walks its contiguous range of tasks with a kPipeStages-deep
// ring of shared-memory tiles: the source tile of task i + kPipeStages is requested with
// cp.async while task i is written out, so the read stream never waits for the writes.
// Tiles are staged in the layout the writes want (transpose mode: pitch tb + 1).
constexpr int kPipeStages = 3;
constexpr int kStageElems = kTileElemsMax + 256;

__device__ __forceinline__ void cp_async_el(double *sm, const double *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(sm)),
               "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async_el(double2 *sm, const double2 *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(sm)),
               "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ double conj_v(double v, bool) { return v; }
__device__ __forceinline__ double2 conj_v(double2 v, bool c) {
  if (c) v.y = -v.y;
  return v;
}

// OFF: the integer type of in-tile offsets (32-bit when every tile's span fits, which keeps
// the per-element address arithmetic to single-word multiply-adds). The records of the CTA's
// tasks (at most kRecCache) are copied to shared memory first, so no task waits on a
// dependent metadata load.
constexpr int kRecCache = 64;

template <typename T, bool CONJ, typename OFF>
__global__ void __launch_bounds__(kThreads)
    treetransform_pipe_kernel(const TaskRec *__restrict__ recs, int64_t ntasks, T *__restrict__ dst,
                              const T *__restrict__ src, CDbl alpha_, CDbl beta_, int beta_zero) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TaskRec rs[kRecCache];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const T alpha = scalar_from<T>(alpha_);
  const T beta = scalar_from<T>(beta_);
  const bool bz = beta_zero != 0;
  pdl_trigger();  // the next kernel may be scheduled; it waits for this grid before reading
  const int64_t per = (ntasks + gridDim.x - 1) / gridDim.x;  // ≤ kRecCache (host)
  const int64_t t_begin = (int64_t)blockIdx.x * per;
  const int64_t t_end = min(ntasks, t_begin + per);
  {
    const int nw = (int)(t_end > t_begin ? t_end - t_begin : 0) * (int)(sizeof(TaskRec) / 8);
    const int64_t *srcw = reinterpret_cast<const int64_t *>(recs + t_begin);
    int64_t *dstw = reinterpret_cast<int64_t *>(rs);
    for (int i = threadIdx.x; i < nw; i += kThreads) dstw[i] = __ldg(srcw + i);
  }
  __syncthreads();
  pdl_wait();  // the records are static; source and destination belong to earlier kernels

  auto issue = [&](int64_t task, T *stage) {
    const TaskRec &R = rs[task - t_begin];
    const int ta = R.ta, tot = R.ta * R.tb, lta = __ffs(R.ta) - 1, ltb = __ffs(R.tb) - 1;
    const OFF sA = (OFF)R.sA, sB = (OFF)R.sB;
    const int na = R.na, nb = R.nb;
    const T *sb = src + R.sbase;
    if (R.mode == 1) {  // source-fast b: coalesced reads, tile stored row-pitched (tb + 1)
      const int pitch = R.tb + 1;
      for (int e = threadIdx.x; e < tot; e += kThreads) {
        const int ia = e >> ltb, ib = e & ((1 << ltb) - 1);
        if (ia < na && ib < nb) cp_async_el(stage + ia * pitch + ib, sb + (OFF)ia * sA + (OFF)ib * sB);
      }
    } else {
      for (int e = threadIdx.x; e < tot; e += kThreads) {
        const int ia = e & (ta - 1), ib = e >> lta;
        if (ia < na && ib < nb) cp_async_el(stage + e, sb + (OFF)ia * sA + (OFF)ib * sB);
      }
    }
  };
  auto write = [&](int64_t task, const T *stage) {
    const TaskRec &R = rs[task - t_begin];
    const int ta = R.ta, tot = R.ta * R.tb, lta = __ffs(R.ta) - 1;
    const int pitch = R.mode == 1 ? R.tb + 1 : 0;
    const OFF dA = (OFF)R.dA, dB = (OFF)R.dB;
    const int na = R.na, nb = R.nb;
    const double u = R.u;
    T *db = dst + R.dbase;
    for (int e0 = 0; e0 < tot; e0 += kThreads * kBatch) {
#pragma unroll
      for (int q = 0; q < kBatch; ++q) {
        const int e = e0 + q * kThreads + threadIdx.x;
        const int ia = e & (ta - 1), ib = e >> lta;  // a fastest: coalesced writes
        if (e < tot && ia < na && ib < nb) {
          const T v = conj_v(stage[pitch ? ia * pitch + ib : e], CONJ);
          T *dp = db + (OFF)ia * dA + (OFF)ib * dB;
          *dp = finish(axpy_r(u, v, zero_val(T{})), alpha, beta, dp, bz);
        }
      }
    }
  };
#pragma unroll
  for (int st = 0; st < kPipeStages; ++st) {
    if (t_begin + st < t_end) issue(t_begin + st, sm + st * kStageElems);
    cp_async_commit();
  }
  int st = 0;
  for (int64_t task = t_begin; task < t_end; ++task) {
    cp_async_wait<kPipeStages - 1>();
    __syncthreads();
    write(task, sm + st * kStageElems);
    __syncthreads();
    if (task + kPipeStages < t_end) issue(task + kPipeStages, sm + st * kStageElems);
    cp_async_commit();
    st = st + 1 == kPipeStages ? 0 : st + 1;
  }
  cp_async_wait<0>();
}

// ---- row-copy kernel for single-tree tables whose groups keep their fastest dim ----------
// Such a transform is a batch of strided row copies (a U(1) or SU(2) permute that leaves the
// leading leg in place: every sub-block row is contiguous on both sides; a small remainder of
// transpose groups rides along with uncoalesced reads). Tiles are exact
// (na × nb, na the full row up to the tile target), so no lane idles on a power-of-two
// round-up, and nothing is staged: each thread issues kBatch loads, then the kBatch scaled
// stores, and the next task's loads follow at once. Row and column come from one multiply-high
// by the precomputed reciprocal `mul` (exact for tile indices below 2¹⁶: Granlund–Montgomery
// division by invariant integers). Without shared-memory tiles the kernel runs at the
// occupancy its registers allow, which keeps enough loads in flight per SM for HBM.
template <typename T, bool CONJ, typename OFF, bool PAIRS>
__global__ void __launch_bounds__(kThreads, (sizeof(T) == 8 && !PAIRS) ? 6 : 4)
    treetransform_rows_kernel(const TaskRec *__restrict__ recs, int64_t ntasks, T *__restrict__ dst,
                              const T *__restrict__ src, CDbl alpha_, CDbl beta_, int beta_zero, int pairs_ok) {
  __shared__ TaskRec rs[kRecCache];
  const T alpha = scalar_from<T>(alpha_);
  const T beta = scalar_from<T>(beta_);
  const bool bz = beta_zero != 0;
  pdl_trigger();  // the next kernel may be scheduled; it waits for this grid before reading
  const int64_t per = (ntasks + gridDim.x - 1) / gridDim.x;  // ≤ kRecCache (host)
  const int64_t t_begin = (int64_t)blockIdx.x * per;
  const int64_t t_end = min(ntasks, t_begin + per);
  {
    const int nw = (int)(t_end > t_begin ? t_end - t_begin : 0) * (int)(sizeof(TaskRec) / 8);
    const int64_t *srcw = reinterpret_cast<const int64_t *>(recs + t_begin);
    int64_t *dstw = reinterpret_cast<int64_t *>(rs);
    for (int i = threadIdx.x; i < nw; i += kThreads) dstw[i] = __ldg(srcw + i);
  }
  __syncthreads();
  pdl_wait();  // the records are static; source and destination belong to earlier kernels

  for (int64_t task = t_begin; task < t_end; ++task) {
    const TaskRec &R = rs[task - t_begin];
    if constexpr (PAIRS) {
      if (R.pairs && pairs_ok) {
        // real rows contiguous on both sides: 16-byte loads and stores of element pairs (half as
        // many per thread and batch: the same bytes in flight)
        const int np = R.na / 2, nun = np * R.nb;
        const uint32_t mul2 = R.mul2;
        const double u = R.u;
        const double2 *sb2 = reinterpret_cast<const double2 *>(src + R.sbase);
        double2 *db2 = reinterpret_cast<double2 *>(dst + R.dbase);
        const OFF sB2 = (OFF)(R.sB / 2), dB2 = (OFF)(R.dB / 2);
        const double a = scalar_from<double>(alpha_), bb = scalar_from<double>(beta_);
        for (int e0 = 0; e0 < nun; e0 += kThreads * kBatchPairs) {
          double2 v[kBatchPairs];
#pragma unroll
          for (int q = 0; q < kBatchPairs; ++q) {
            const int e = e0 + q * kThreads + threadIdx.x;
            const int row = mul2 ? (int)__umulhi((unsigned)e, mul2) : e, cp = e - row * np;
            if (e < nun) v[q] = __ldg(sb2 + (OFF)cp + (OFF)row * sB2);
          }
#pragma unroll
          for (int q = 0; q < kBatchPairs; ++q) {
            const int e = e0 + q * kThreads + threadIdx.x;
            const int row = mul2 ? (int)__umulhi((unsigned)e, mul2) : e, cp = e - row * np;
            if (e < nun) {
              double2 *dp = db2 + (OFF)cp + (OFF)row * dB2;
              double2 r = make_double2(a * (u * v[q].x), a * (u * v[q].y));
              if (!bz) {
                const double2 o = *dp;
                r.x = fma(bb, o.x, r.x);
                r.y = fma(bb, o.y, r.y);
              }
              *dp = r;
            }
          }
        }
        continue;
      }
    }
    const int na = R.na, nel = R.na * R.nb;
    const uint32_t mul = R.mul;
    const OFF sA = (OFF)R.sA, sB = (OFF)R.sB, dA = (OFF)R.dA, dB = (OFF)R.dB;
    const double u = R.u;
    const T *sb = src + R.sbase;
    T *db = dst + R.dbase;
    for (int e0 = 0; e0 < nel; e0 += kThreads * kBatch) {
      T v[kBatch];
#pragma unroll
      for (int q = 0; q < kBatch; ++q) {
        const int e = e0 + q * kThreads + threadIdx.x;
        const int row = mul ? (int)__umulhi((unsigned)e, mul) : e, col = e - row * na;
        if (e < nel) v[q] = ld_val(sb + (OFF)col * sA + (OFF)row * sB, CONJ);
      }
#pragma unroll
      for (int q = 0; q < kBatch; ++q) {
        const int e = e0 + q * kThreads + threadIdx.x;
        const int row = mul ? (int)__umulhi((unsigned)e, mul) : e, col = e - row * na;
        if (e < nel) {
          T *dp = db + (OFF)col * dA + (OFF)row * dB;
          *dp = finish(axpy_r(u, v[q], zero_val(T{})), alpha, beta, dp, bz);
        }
      }
    }
  }
}

// TKB_TRANSFORM_KERNEL selects a kernel for comparison: "plain" the non-pipelined kernel for
// every table, "pipe" the staged ring for every single-tree table (no row-copy kernel)
bool use_plain_transform() {
  const char *e = std::getenv("TKB_TRANSFORM_KERNEL");
  return e && std::strcmp(e, "plain") == 0;
}
bool use_pipe_transform() {
  const char *e = std::getenv("TKB_TRANSFORM_KERNEL");
  return e && std::strcmp(e, "pipe") == 0;
}

int64_t pow2ceil(int64_t x) {
  int64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

// CTAs per SM of a kernel launched with `threads` threads and `smem` bytes of dynamic shared
// memory: the shared-memory attribute is set and the occupancy queried once per kernel and
// device (each kernel has one launch shape), so eager launches make no attribute calls
int tkb_occupancy(int device, const void *kfn, int threads, size_t smem) {
  static std::mutex mu;
  static std::unordered_map<const void *, int> cache[64];
  if (device < 0 || device >= 64) return 0;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache[device].find(kfn);
  if (it != cache[device].end()) return it->second;
  if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem) != cudaSuccess) return 0;
  cache[device][kfn] = per_sm;
  return per_sm;
}

extern "C" int tkb_table_create(tkb_ctx *ctx, const tkb_table_desc *d, tkb_table **out) {
  if (!ctx || !d || !out) return TKB_ERR_ARG;
  *out = nullptr;
  const int N = d->nind;
  if (N < 0 || N > TKB_MAX_IND) return tkb_set_error(ctx, TKB_ERR_ARG, "nind out of range");
  if (d->ngroups < 0) return tkb_set_error(ctx, TKB_ERR_ARG, "negative ngroups");
  {
    std::vector<int> seen(N, 0);
    for (int k = 0; k < N; ++k) {
      if (d->perm[k] < 0 || d->perm[k] >= N || seen[d->perm[k]]++)
        return tkb_set_error(ctx, TKB_ERR_ARG, "perm is not a permutation");
    }
  }
  const int64_t G = d->ngroups;
  if (G > 0 && (!d->group_src_ptr || !d->group_dst_ptr || !d->coeff_ptr || !d->coeffs ||
                (N > 0 && (!d->sizes || !d->src_strides || !d->dst_strides)) ||
                !d->src_offsets || !d->dst_offsets))
    return tkb_set_error(ctx, TKB_ERR_ARG, "null table array");

  std::vector<TGroup> hg;
  hg.reserve(G);
  std::vector<int64_t> hsstr, hsoff, hdstr, hdoff;
  std::vector<int32_t> htask;  // task → group
  std::vector<int32_t> hidx;   // task → (tile a, tile b, outer multi-index)
  std::vector<TaskRec> hrec;   // task → tree-0 bases and extents (single-tree tables)
  std::vector<TaskRec> hrow;   // exact row tiles (single-tree tables, every group mode 0)
  bool all_off32 = true, all_rows = true, row_off32 = true;
  int64_t row_pair_elems = 0;  // elements of row tasks that can be copied in 16-byte pairs
  int64_t row_transposed = 0;  // elements of transpose groups in the row tiles
  std::vector<double> hcoef;
  int64_t ntasks = 0, er = 0, ew = 0;
  size_t smem_max_f64 = 0, smem_max_c128 = 0;
  int max_trees = 1, max_dst = 1;
  // tile target: 2048 elements per task, smaller when the whole transform would not give
  // every SM about four tasks (small permutes are latency-bound, not bandwidth-bound)
  int64_t kTileElems = kTileElemsMax, kRowTileElems = kTileElemsMax;
  {
    int64_t total = 0;
    for (int64_t g = 0; g < G; ++g) {
      int64_t vol = 1;
      for (int k = 0; k < N; ++k) vol *= std::max<int64_t>(1, d->sizes[g * N + k]);
      total += vol * (d->group_dst_ptr[g + 1] - d->group_dst_ptr[g]);
    }
    while (kTileElems > 256 && total / kTileElems < (int64_t)ctx->num_sms * 4) kTileElems >>= 1;
    // row tiles: about two per SM at least; a row task costs a fixed record fetch and one load
    // round trip, so small transforms run faster with fewer, larger row tasks
    while (kRowTileElems > 256 && total / kRowTileElems < (int64_t)ctx->num_sms * 2) kRowTileElems >>= 1;
  }

  for (int64_t g = 0; g < G; ++g) {
    const int64_t s0 = d->group_src_ptr[g], s1 = d->group_src_ptr[g + 1];
    const int64_t t0 = d->group_dst_ptr[g], t1 = d->group_dst_ptr[g + 1];
    const int64_t c0 = d->coeff_ptr[g], c1 = d->coeff_ptr[g + 1];
    const int64_t nsrc = s1 - s0, ndst = t1 - t0;
    if (nsrc <= 0 || ndst <= 0 || c1 - c0 != nsrc * ndst)
      return tkb_set_error(ctx, TKB_ERR_ARG, "inconsistent group pointers");
    const int64_t *sz = d->sizes + g * N;
    int64_t vol = 1;
    for (int k = 0; k < N; ++k) {
      if (sz[k] <= 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "non-positive sub-block size");
      vol *= sz[k];
    }
    // bounds validation of every tree (prevents any out-of-range device access)
    for (int64_t j = s0; j < s1; ++j) {
      int64_t hi = d->src_offsets[j];
      if (hi < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative source offset");
      for (int k = 0; k < N; ++k) {
        const int64_t st = d->src_strides[j * N + k];
        if (st < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative source stride");
        hi += (sz[k] - 1) * st;
      }
      if (hi >= d->src_len)
        return tkb_set_error(ctx, TKB_ERR_SIZE, "source sub-block exceeds source data length");
    }
    for (int64_t i = t0; i < t1; ++i) {
      int64_t hi = d->dst_offsets[i];
      if (hi < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative destination offset");
      for (int k = 0; k < N; ++k) {
        const int64_t st = d->dst_strides[i * N + k];
        if (st < 0) return tkb_set_error(ctx, TKB_ERR_SIZE, "negative destination stride");
        hi += (sz[d->perm[k]] - 1) * st;
      }
      if (hi >= d->dst_len)
        return tkb_set_error(ctx, TKB_ERR_SIZE,
                             "destination sub-block exceeds destination data length");
    }
    er += vol * nsrc;
    ew += vol * ndst;

    // canonical dims in destination order: (size, src strides per tree, dst strides per tree)
    struct Dim {
      int64_t size;
      std::vector<int64_t> ss, ds;
    };
    std::vector<Dim> dims;
    for (int k = 0; k < N; ++k) {
      const int ks = d->perm[k];
      if (sz[ks] == 1) continue;
      Dim dm;
      dm.size = sz[ks];
      for (int64_t j = s0; j < s1; ++j) dm.ss.push_back(d->src_strides[j * N + ks]);
      for (int64_t i = t0; i < t1; ++i) dm.ds.push_back(d->dst_strides[i * N + k]);
      dims.push_back(dm);
    }
    // merge neighbours contiguous on both sides for every tree
    for (size_t k = 0; k + 1 < dims.size();) {
      bool ok = true;
      for (size_t j = 0; j < dims[k].ss.size() && ok; ++j)
        ok = dims[k + 1].ss[j] == dims[k].ss[j] * dims[k].size;
      for (size_t i = 0; i < dims[k].ds.size() && ok; ++i)
        ok = dims[k + 1].ds[i] == dims[k].ds[i] * dims[k].size;
      if (ok) {
        dims[k].size *= dims[k + 1].size;
        dims.erase(dims.begin() + k + 1);
      } else {
        ++k;
      }
    }
    if (dims.empty()) {  // scalar sub-block
      Dim dm;
      dm.size = 1;
      dm.ss.assign(nsrc, 1);
      dm.ds.assign(ndst, 1);
      dims.push_back(dm);
    }
    const int nd = (int)dims.size();
    TGroup tg;
    std::memset(&tg, 0, sizeof(tg));
    tg.ndim = nd;
    for (int k = 0; k < nd; ++k) {
      if (dims[k].size > INT32_MAX)
        return tkb_set_error(ctx, TKB_ERR_UNSUPPORTED, "sub-block dimension beyond 2^31 elements");
      tg.size[k] = dims[k].size;
    }
    // fastest dims (tree 0 pattern; all trees of a group share it)
    int fa = 0, fs = 0;
    for (int k = 1; k < nd; ++k) {
      if (dims[k].ds[0] < dims[fa].ds[0]) fa = k;
      if (dims[k].ss[0] < dims[fs].ss[0]) fs = k;
    }
    const size_t el64 = 8, el128 = 16;
    int64_t ta, tb;
    int db;
    if (fa == fs) {
      tg.mode = 0;
      db = -1;
      int64_t best = 0;
      for (int k = 0; k < nd; ++k)
        if (k != fa && dims[k].size > best) { best = dims[k].size; db = k; }
      ta = std::min<int64_t>(pow2ceil(dims[fa].size), kTileElems);
      tb = db >= 0 ? std::min<int64_t>(pow2ceil(dims[db].size), std::max<int64_t>(1, kTileElems / ta)) : 1;
      // shared-memory budget when several trees are staged
      while (nsrc > 1 && (size_t)(nsrc * ta * tb) * el128 > kSmemBudget && (ta > 1 || tb > 1)) {
        if (tb > 1) tb >>= 1; else ta >>= 1;
      }
    } else {
      tg.mode = 1;
      db = fs;
      ta = std::min<int64_t>(pow2ceil(dims[fa].size), 32);
      tb = std::min<int64_t>(pow2ceil(dims[db].size), 32);
      while (ta * tb < kTileElems) {
        const bool grow_a = ta < dims[fa].size && (ta <= tb || tb >= dims[db].size);
        const bool grow_b = tb < dims[db].size;
        if (grow_a && ta < 256) ta <<= 1;
        else if (grow_b && tb < 256) tb <<= 1;
        else break;
      }
      while ((size_t)(nsrc * ta * (tb + 1)) * el128 > kSmemBudget && (ta > 1 || tb > 1)) {
        if (ta >= tb && ta > 1) ta >>= 1; else tb >>= 1;
      }
    }
    tg.da = fa;
    tg.db = db;
    tg.ta = (int)ta;
    tg.tb = (int)tb;
    tg.nouter = 0;
    int64_t nouter_total = 1;
    for (int k = 0; k < nd; ++k) {
      if (k == fa || k == db) continue;
      tg.outer[tg.nouter++] = k;
      nouter_total *= dims[k].size;
    }
    tg.ntile_a = (dims[fa].size + ta - 1) / ta;
    tg.ntile_b = db >= 0 ? (dims[db].size + tb - 1) / tb : 1;
    tg.task_begin = ntasks;
    ntasks += tg.ntile_a * tg.ntile_b * nouter_total;
    tg.src_tree_begin = (int64_t)hsoff.size();
    tg.dst_tree_begin = (int64_t)hdoff.size();
    tg.nsrc = nsrc;
    tg.ndst = ndst;
    tg.coeff_begin = (int64_t)hcoef.size();
    for (int64_t j = 0; j < nsrc; ++j) {
      hsoff.push_back(d->src_offsets[s0 + j]);
      for (int k = 0; k < TKB_MAX_IND; ++k) hsstr.push_back(k < nd ? dims[k].ss[j] : 0);
    }
    for (int64_t i = 0; i < ndst; ++i) {
      hdoff.push_back(d->dst_offsets[t0 + i]);
      for (int k = 0; k < TKB_MAX_IND; ++k) hdstr.push_back(k < nd ? dims[k].ds[i] : 0);
    }
    for (int64_t c = c0; c < c1; ++c) hcoef.push_back(d->coeffs[c]);
    const bool staged = !(tg.mode == 0 && nsrc == 1 && ndst == 1);
    if (staged) {
      const int64_t te = tg.mode == 1 ? ta * (tb + 1) : ta * tb;
      smem_max_f64 = std::max(smem_max_f64, (size_t)(nsrc * te) * el64);
      smem_max_c128 = std::max(smem_max_c128, (size_t)(nsrc * te) * el128);
    }
    max_trees = std::max<int>(max_trees, (int)nsrc);
    max_dst = std::max<int>(max_dst, (int)ndst);
    tg.sa0 = dims[fa].ss[0];
    tg.da0 = dims[fa].ds[0];
    tg.sb0 = db >= 0 ? dims[db].ss[0] : 0;
    tg.db0 = db >= 0 ? dims[db].ds[0] : 0;
    tg.u0 = d->coeffs[c0];
    {
      const int64_t lim = (int64_t)INT32_MAX;
      const int64_t so = (ta - 1) * tg.sa0 + (tb - 1) * tg.sb0, dso = (ta - 1) * tg.da0 + (tb - 1) * tg.db0;
      if (tg.sa0 > lim || tg.sb0 > lim || tg.da0 > lim || tg.db0 > lim || so > lim || dso > lim) all_off32 = false;
    }
    htask.insert(htask.end(), (size_t)(ntasks - tg.task_begin), (int32_t)g);
    for (int64_t t = 0; t < ntasks - tg.task_begin; ++t) {
      int64_t r = t;
      int32_t w[kTaskWords] = {0};
      w[1] = (int32_t)(r % tg.ntile_b);
      r /= tg.ntile_b;
      w[0] = (int32_t)(r % tg.ntile_a);
      r /= tg.ntile_a;
      for (int q = 0; q < tg.nouter; ++q) {
        const int64_t sq = tg.size[tg.outer[q]];
        w[2 + q] = (int32_t)(r % sq);
        r /= sq;
      }
      hidx.insert(hidx.end(), w, w + kTaskWords);
      if (nsrc == 1 && ndst == 1) {
        const int64_t a0 = (int64_t)w[0] * ta, b0 = (int64_t)w[1] * tb;
        TaskRec rec;
        rec.sbase = d->src_offsets[s0] + a0 * tg.sa0 + b0 * tg.sb0;
        rec.dbase = d->dst_offsets[t0] + a0 * tg.da0 + b0 * tg.db0;
        for (int q = 0; q < tg.nouter; ++q) {
          rec.sbase += (int64_t)w[2 + q] * dims[tg.outer[q]].ss[0];
          rec.dbase += (int64_t)w[2 + q] * dims[tg.outer[q]].ds[0];
        }
        const int64_t sa = dims[fa].size, sb = db >= 0 ? dims[db].size : 1;
        rec.na = (int32_t)std::min<int64_t>(ta, sa - a0);
        rec.nb = (int32_t)std::min<int64_t>(tb, sb - b0);
        rec.sA = tg.sa0;
        rec.sB = tg.sb0;
        rec.dA = tg.da0;
        rec.dB = tg.db0;
        rec.u = tg.u0;
        rec.ta = (int32_t)ta;
        rec.tb = (int32_t)tb;
        rec.mode = tg.mode;
        rec.mul = 0;
        hrec.push_back(rec);
      }
    }
    if (nsrc == 1 && ndst == 1 && all_rows) {
      // exact row tiles: ra elements of the destination's fast dim (the whole row up to the
      // tile target) times rb rows of the tile's b dim (the largest other dim; for a transpose
      // group the source's fast dim, read uncoalesced); a fastest, then b, then the outer dims
      if (tg.mode == 1) row_transposed += vol;
      const int64_t L = dims[fa].size, LB = db >= 0 ? dims[db].size : 1;
      const int64_t ra = std::min<int64_t>(L, kRowTileElems);
      const int64_t rb = std::max<int64_t>(1, std::min<int64_t>(LB, kRowTileElems / ra));
      const int64_t nra = (L + ra - 1) / ra, nrb = (LB + rb - 1) / rb;
      {
        const int64_t lim = (int64_t)INT32_MAX;
        const int64_t so = (ra - 1) * tg.sa0 + (rb - 1) * tg.sb0, dso = (ra - 1) * tg.da0 + (rb - 1) * tg.db0;
        if (tg.sa0 > lim || tg.sb0 > lim || tg.da0 > lim || tg.db0 > lim || so > lim || dso > lim) row_off32 = false;
      }
      for (int64_t o = 0; o < nouter_total; ++o) {
        int64_t r = o, sbo = d->src_offsets[s0], dbo = d->dst_offsets[t0];
        for (int q = 0; q < tg.nouter; ++q) {
          const Dim &dq = dims[tg.outer[q]];
          const int64_t i = r % dq.size;
          r /= dq.size;
          sbo += i * dq.ss[0];
          dbo += i * dq.ds[0];
        }
        for (int64_t ib = 0; ib < nrb; ++ib) {
          for (int64_t ia = 0; ia < nra; ++ia) {
            const int64_t a0 = ia * ra, b0 = ib * rb;
            TaskRec rec;
            rec.sbase = sbo + a0 * tg.sa0 + b0 * tg.sb0;
            rec.dbase = dbo + a0 * tg.da0 + b0 * tg.db0;
            rec.na = (int32_t)std::min<int64_t>(ra, L - a0);
            rec.nb = (int32_t)std::min<int64_t>(rb, LB - b0);
            rec.sA = tg.sa0;
            rec.sB = tg.sb0;
            rec.dA = tg.da0;
            rec.dB = tg.db0;
            rec.u = tg.u0;
            rec.ta = rec.na;
            rec.tb = rec.nb;
            rec.mode = 0;
            rec.mul = rec.na > 1 ? 0xFFFFFFFFu / (uint32_t)rec.na + 1u : 0u;
            // 16-byte pairs: contiguous rows on both sides, even row length and even row starts
            rec.pairs = (tg.mode == 0 && rec.sA == 1 && rec.dA == 1 && rec.na % 2 == 0 && rec.sbase % 2 == 0 &&
                         rec.dbase % 2 == 0 && (rec.nb == 1 || (rec.sB % 2 == 0 && rec.dB % 2 == 0)))
                            ? 1
                            : 0;
            rec.mul2 = rec.na > 2 ? 0xFFFFFFFFu / (uint32_t)(rec.na / 2) + 1u : 0u;
            if (rec.pairs) row_pair_elems += (int64_t)rec.na * rec.nb;
            hrow.push_back(rec);
          }
        }
      }
    } else {
      all_rows = false;
    }
    hg.push_back(tg);
  }
  if (std::max(smem_max_f64, smem_max_c128) > ctx->smem_optin)
    return tkb_set_error(ctx, TKB_ERR_UNSUPPORTED, "fusion block too large for shared memory");

  tkb_table *t = new tkb_table();
  t->owner = ctx;
  t->ngroups = (int)G;
  t->ntasks = ntasks;
  t->elems_read = er;
  t->elems_written = ew;
  t->max_trees = max_trees;
  t->single_tree = max_trees == 1 && max_dst == 1;
  t->off32 = all_off32;
  // the row kernel takes the table when its transpose groups are a small remainder (sub-blocks
  // whose leading leg has dimension 1, for example); otherwise the staged ring transposes
  if (t->single_tree && all_rows && row_off32 && row_transposed * 64 <= er) t->nrow_tasks = (int64_t)hrow.size();
  t->row_pair_elems = row_pair_elems;
  t->smem_f64 = smem_max_f64;
  t->smem_c128 = smem_max_c128;
  t->src_len = d->src_len;
  t->dst_len = d->dst_len;
  auto up = [&](void **dptr, const void *h, size_t bytes) -> cudaError_t {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(dptr, bytes);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dptr, h, bytes, cudaMemcpyHostToDevice);
  };
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = up((void **)&t->groups, hg.data(), hg.size() * sizeof(TGroup));
  if (e == cudaSuccess) e = up((void **)&t->task_group, htask.data(), htask.size() * 4);
  if (e == cudaSuccess) e = up((void **)&t->task_idx, hidx.data(), hidx.size() * 4);
  if (e == cudaSuccess && t->single_tree) e = up((void **)&t->task_rec, hrec.data(), hrec.size() * sizeof(TaskRec));
  if (e == cudaSuccess && t->nrow_tasks > 0)
    e = up((void **)&t->row_rec, hrow.data(), hrow.size() * sizeof(TaskRec));
  if (e == cudaSuccess) e = up((void **)&t->sstr, hsstr.data(), hsstr.size() * 8);
  if (e == cudaSuccess) e = up((void **)&t->soff, hsoff.data(), hsoff.size() * 8);
  if (e == cudaSuccess) e = up((void **)&t->dstr, hdstr.data(), hdstr.size() * 8);
  if (e == cudaSuccess) e = up((void **)&t->doff, hdoff.data(), hdoff.size() * 8);
  if (e == cudaSuccess) e = up((void **)&t->coeffs, hcoef.data(), hcoef.size() * 8);
  if (e != cudaSuccess) {
    tkb_table_destroy(t);
    return tkb_set_error(ctx, e == cudaErrorMemoryAllocation ? TKB_ERR_OOM : TKB_ERR_CUDA,
                         std::string("table upload: ") + cudaGetErrorString(e));
  }
  *out = t;
  return TKB_OK;
}

extern "C" int tkb_table_destroy(tkb_table *t) {
  if (!t) return TKB_OK;
  cudaFree(t->groups);
  cudaFree(t->task_group);
  cudaFree(t->task_idx);
  cudaFree(t->task_rec);
  cudaFree(t->row_rec);
  cudaFree(t->sstr);
  cudaFree(t->soff);
  cudaFree(t->dstr);
  cudaFree(t->doff);
  cudaFree(t->coeffs);
  delete t;
  return TKB_OK;
}

extern "C" int tkb_table_info(const tkb_table *t, int64_t *ntasks, int64_t *er, int64_t *ew) {
  if (!t) return TKB_ERR_ARG;
  if (ntasks) *ntasks = t->ntasks;
  if (er) *er = t->elems_read;
  if (ew) *ew = t->elems_written;
  return TKB_OK;
}

int tkb_transform_launch(tkb_ctx *ctx, const tkb_table *t, int dtype, void *dst,
                         const void *src, tkb_scalar alpha, tkb_scalar beta, int conj) {
  if (t->ntasks == 0) return TKB_OK;
  const int grid = (int)std::min<int64_t>(t->ntasks, (int64_t)ctx->num_sms * 16);
  CDbl a{alpha.re, alpha.im}, b{beta.re, beta.im};
  const int bz = (beta.re == 0.0 && beta.im == 0.0) ? 1 : 0;
  if (t->nrow_tasks > 0 && (dtype == TKB_F64 || dtype == TKB_C128) && !use_plain_transform() &&
      !use_pipe_transform()) {
    if (dtype == TKB_F64 && (alpha.im != 0.0 || beta.im != 0.0))
      return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
    // persistent CTAs: as many as reside at once, with at most kRecCache tasks each
    using KD = void (*)(const TaskRec *, int64_t, double *, const double *, CDbl, CDbl, int, int);
    using KC = void (*)(const TaskRec *, int64_t, double2 *, const double2 *, CDbl, CDbl, int, int);
    KD kd = nullptr;
    KC kc = nullptr;
    const void *kfn;
    // 16-byte pair accesses need 16-byte aligned data vectors
    const int pairs_ok = ((((uintptr_t)dst | (uintptr_t)src) & 15) == 0) ? 1 : 0;
    if (dtype == TKB_F64) {
      // the kernel with the 16-byte pair path (fewer resident CTAs) when most of the table can
      // use it, else the scalar one
      kd = (pairs_ok && t->row_pair_elems * 2 >= t->elems_read) ? treetransform_rows_kernel<double, false, int32_t, true>
                                                                : treetransform_rows_kernel<double, false, int32_t, false>;
      kfn = (const void *)kd;
    } else {
      kc = conj ? treetransform_rows_kernel<double2, true, int32_t, false>
                : treetransform_rows_kernel<double2, false, int32_t, false>;
      kfn = (const void *)kc;
    }
    const int per_sm = tkb_occupancy(ctx->device, kfn, kThreads, 0);
    if (per_sm <= 0) return tkb_set_error(ctx, TKB_ERR_CUDA, "row transform: occupancy query failed");
    const int64_t nt = t->nrow_tasks;
    int64_t pg = std::min<int64_t>(nt, (int64_t)ctx->num_sms * per_sm);
    pg = std::max<int64_t>(pg, (nt + kRecCache - 1) / kRecCache);
    if (kd)
      TKB_CUDA_TRY(ctx, launch_pdl(kd, dim3((int)pg), dim3(kThreads), 0, ctx->stream, t->row_rec, nt,
                                   (double *)dst, (const double *)src, a, b, bz, pairs_ok));
    else
      TKB_CUDA_TRY(ctx, launch_pdl(kc, dim3((int)pg), dim3(kThreads), 0, ctx->stream, t->row_rec, nt,
                                   (double2 *)dst, (const double2 *)src, a, b, bz, pairs_ok));
    ctx->launches++;
    TKB_CUDA_TRY(ctx, cudaGetLastError());
    return TKB_OK;
  }
  if (t->single_tree && (dtype == TKB_F64 || dtype == TKB_C128) && !use_plain_transform()) {
    if (dtype == TKB_F64 && (alpha.im != 0.0 || beta.im != 0.0))
      return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
    // persistent CTAs: as many as reside at once (occupancy of the stage ring), with at most
    // kRecCache tasks each
    const size_t el = dtype == TKB_F64 ? 8 : 16;
    const size_t smem = (size_t)kPipeStages * kStageElems * el;
    using KD = void (*)(const TaskRec *, int64_t, double *, const double *, CDbl, CDbl, int);
    using KC = void (*)(const TaskRec *, int64_t, double2 *, const double2 *, CDbl, CDbl, int);
    KD kd = nullptr;
    KC kc = nullptr;
    const void *kfn;
    if (dtype == TKB_F64) {
      kd = t->off32 ? treetransform_pipe_kernel<double, false, int32_t> : treetransform_pipe_kernel<double, false, int64_t>;
      kfn = (const void *)kd;
    } else {
      kc = conj ? (t->off32 ? treetransform_pipe_kernel<double2, true, int32_t>
                            : treetransform_pipe_kernel<double2, true, int64_t>)
                : (t->off32 ? treetransform_pipe_kernel<double2, false, int32_t>
                            : treetransform_pipe_kernel<double2, false, int64_t>);
      kfn = (const void *)kc;
    }
    const int per_sm = tkb_occupancy(ctx->device, kfn, kThreads, smem);
    if (per_sm <= 0) return tkb_set_error(ctx, TKB_ERR_CUDA, "pipelined transform: occupancy query failed");
    int64_t pg = std::min<int64_t>(t->ntasks, (int64_t)ctx->num_sms * std::max(1, per_sm));
    pg = std::max<int64_t>(pg, (t->ntasks + kRecCache - 1) / kRecCache);
    const int pgrid = (int)pg;
    if (kd)
      TKB_CUDA_TRY(ctx, launch_pdl(kd, dim3(pgrid), dim3(kThreads), smem, ctx->stream, t->task_rec, t->ntasks,
                                   (double *)dst, (const double *)src, a, b, bz));
    else
      TKB_CUDA_TRY(ctx, launch_pdl(kc, dim3(pgrid), dim3(kThreads), smem, ctx->stream, t->task_rec, t->ntasks,
                                   (double2 *)dst, (const double2 *)src, a, b, bz));
    ctx->launches++;
    TKB_CUDA_TRY(ctx, cudaGetLastError());
    return TKB_OK;
  }
  if (dtype == TKB_F64) {
    if (alpha.im != 0.0 || beta.im != 0.0)
      return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
    const size_t smem = t->smem_f64;
    auto k = treetransform_kernel<double, false>;
    if (smem > 48 * 1024) TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TKB_CUDA_TRY(ctx, launch_pdl(k, dim3(grid), dim3(kThreads), smem, ctx->stream, t->groups, t->task_group,
                                 t->task_idx, t->ntasks, t->sstr, t->soff, t->dstr, t->doff, t->coeffs,
                                 (double *)dst, (const double *)src, a, b, bz));
  } else if (dtype == TKB_C128) {
    const size_t smem = t->smem_c128;
    auto k = conj ? treetransform_kernel<double2, true> : treetransform_kernel<double2, false>;
    if (smem > 48 * 1024) TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TKB_CUDA_TRY(ctx, launch_pdl(k, dim3(grid), dim3(kThreads), smem, ctx->stream, t->groups, t->task_group,
                                 t->task_idx, t->ntasks, t->sstr, t->soff, t->dstr, t->doff, t->coeffs,
                                 (double2 *)dst, (const double2 *)src, a, b, bz));
  } else {
    return tkb_set_error(ctx, TKB_ERR_ARG, "unknown dtype");
  }
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}
