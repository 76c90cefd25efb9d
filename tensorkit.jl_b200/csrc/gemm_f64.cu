// Plain FP64 / ComplexF64 grouped block GEMM: one launch for all coupled-sector blocks of a
// TensorKit mul! (src/tensors/linalg.jl:330-370).
//
// Tensor path: FP64 DMMA (mma.sync m16n8k8 for real data, m8n8k4 for complex). tcgen05 has no
// f64 kind, so the double-precision tensor pipe is reached through DMMA; the split-precision
// path (gemm_split.cu) is the tcgen05 one.
//
// Work decomposition: 64×64 output tiles; when the tiles would leave resident CTA slots idle,
// the K loops of the longest tiles are cut into pieces (split K) so that the pieces fill about
// one wave. Tasks (tile, K range) are sorted by decreasing length and dealt round-robin to the
// CTAs of the launch (a static, cost-ordered queue: no atomics to claim work). A piece of a split
// tile stores its FP64 partial tile; the piece that arrives last on the tile's counter adds all
// partials in piece order (deterministic, no piece waits for another) and applies α, β.
//
// Real CTA: 4 warps in a 2×2 grid (each 32×32 = 2×4 m16n8k8 tiles, two accumulator sets: one
// per K sub-step of 8), BK = 16, a three-stage cp.async ring (two stages in flight while one is
// consumed; one barrier per K step; a stage's DMMA are issued before the refill copies).
// Operand tiles are copied in 16-byte pairs when the block's layout keeps pairs aligned (op N,
// even offsets and leading dimensions, 16-byte aligned base), else in 8-byte elements; elements
// outside the block are zero-filled, so any lda/offset parity works. Complex blocks copy whole
// 16-byte elements and issue four real DMMA per fragment pair.
//
// What bounds it: the DMMA pipe runs m16n8k8 at 64 cycles per SM sub-partition (37 TFLOP/s
// measured on B200); the per-thread cp.async copies of a 16 KB stage cost the SM about a third
// of that again (per-instruction load/store-unit work), so large blocks reach about 30 TFLOP/s.
#include <algorithm>
#include <cstring>

#include "tkb_internal.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NST = 3;
constexpr int APAD = 4, BPAD = 4;      // real: keeps 16-byte row alignment, spreads banks
constexpr int CAPAD = 2, CBPAD = 2;    // complex (16-byte elements)
constexpr int kRealThreads = 128, kCplxThreads = 256;

struct CDbl {
  double x, y;
};

// one task of the plain kernels: a 64×64 output tile and a range of its K steps
struct PTask {
  int32_t block, m0, n0, kind;  // kind 0: products, 1: β-scale only (k = 0)
  int32_t kb, ke;               // K steps [kb, ke) of BK
  int32_t slot, nsplit;         // split K: counter slot, pieces of the tile (1 = unsplit)
  int32_t sid, pbase;           // piece index, first partial buffer of the tile
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
// 16-byte copy of which the first `bytes` (0, 8 or 16) come from global memory, the rest zero
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Timeline build (-DTKB_TIMELINE): per CTA of the real kernel, global-timer stamps (ns) at entry
// (0), after the grid-dependency wait (1), after the first task's K loop (2) and split-K
// arrival (3), at exit (4); slot 5 counts the CTA's tasks, slot 6 holds the first task's
// pieces and whether it was the last to arrive (2·nsplit + last). Read with
// tkb_timeline_read_plain; the default build compiles every stamp away.
#ifdef TKB_TIMELINE
constexpr int kPlTlCtas = 512, kPlTlSlots = 8;
__device__ unsigned long long tkb_tl_plain[kPlTlCtas * kPlTlSlots];
__device__ __forceinline__ unsigned long long pl_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
#define PL_SET(k, v)                                                                         \
  do {                                                                                       \
    if (threadIdx.x == 0 && blockIdx.x < kPlTlCtas) tkb_tl_plain[blockIdx.x * kPlTlSlots + (k)] = (v); \
  } while (0)
#else
#define PL_SET(k, v) ((void)0)
#endif
#define PL_STAMP(k) PL_SET(k, pl_now())

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
// D(16×8) += A(16×8) B(8×8), FP64. Lane (g = lane/4, t = lane%4): a = A[g][t], A[g+8][t],
// A[g][t+4], A[g+8][t+4]; b = B[t][g], B[t+4][g]; c = D[g][2t], D[g][2t+1], D[g+8][2t],
// D[g+8][2t+1] (checked against a host product on the device)
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// ---- real ----------------------------------------------------------------------------
struct SmemR {
  double A[NST][BK][BM + APAD];  // op(A) tile, [k][row]
  double B[NST][BN][BK + BPAD];  // op(B) tile, [col][k]
};

// vec: bit 0 = A tiles as 16-byte pairs, bit 1 = B tiles as 16-byte pairs
__device__ __forceinline__ void load_tiles_r(SmemR &s, int st, const GBlock &b, const double *A,
                                             const double *B, int64_t m0, int64_t n0, int64_t k0, int vec) {
  const int tid = threadIdx.x;
  if (vec & 1) {  // op N, pairs of rows: 32 pairs × BK columns
#pragma unroll
    for (int r = 0; r < (BM * BK) / (2 * kRealThreads); ++r) {
      const int e = tid + r * kRealThreads;
      const int i2 = e % (BM / 2), l = e / (BM / 2);
      const int64_t gi = m0 + 2 * i2, gl = k0 + l;
      const int bytes = (gl < b.k && gi < b.m) ? (gi + 1 < b.m ? 16 : 8) : 0;
      const double *p = A + b.offA + (bytes ? gi + gl * b.lda : 0);
      cp_async16(&s.A[st][l][2 * i2], p, bytes);
    }
  } else if (b.opA == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BM * BK) / kRealThreads; ++r) {
      const int e = tid + r * kRealThreads;
      const int i = e % BM, l = e / BM;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      cp_async8(&s.A[st][l][i], A + b.offA + (ok ? gi + gl * b.lda : 0), ok);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BM * BK) / kRealThreads; ++r) {
      const int e = tid + r * kRealThreads;
      const int l = e % BK, i = e / BK;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      cp_async8(&s.A[st][l][i], A + b.offA + (ok ? gl + gi * b.lda : 0), ok);
    }
  }
  if (vec & 2) {  // op N, pairs along K: BK/2 pairs × BN columns
#pragma unroll
    for (int r = 0; r < (BN * BK) / (2 * kRealThreads); ++r) {
      const int e = tid + r * kRealThreads;
      const int l2 = e % (BK / 2), j = e / (BK / 2);
      const int64_t gl = k0 + 2 * l2, gj = n0 + j;
      const int bytes = (gj < b.n && gl < b.k) ? (gl + 1 < b.k ? 16 : 8) : 0;
      const double *p = B + b.offB + (bytes ? gl + gj * b.ldb : 0);
      cp_async16(&s.B[st][j][2 * l2], p, bytes);
    }
  } else if (b.opB == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BN * BK) / kRealThreads; ++r) {
      const int e = tid + r * kRealThreads;
      const int l = e % BK, j = e / BK;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      cp_async8(&s.B[st][j][l], B + b.offB + (ok ? gl + gj * b.ldb : 0), ok);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BN * BK) / kRealThreads; ++r) {
      const int e = tid + r * kRealThreads;
      const int j = e % BN, l = e / BN;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      cp_async8(&s.B[st][j][l], B + b.offB + (ok ? gj + gl * b.ldb : 0), ok);
    }
  }
}

// 16-byte pairs are usable for an operand in op N whose offset and leading dimension are even
// (the base pointer's alignment is checked at launch)
__device__ __forceinline__ int vec_flags(const GBlock &b, int base_ok) {
  int v = 0;
  if ((base_ok & 1) && b.opA == TKB_OP_N && !(b.offA & 1) && !(b.lda & 1)) v |= 1;
  if ((base_ok & 2) && b.opB == TKB_OP_N && !(b.offB & 1) && !(b.ldb & 1)) v |= 2;
  return v;
}

// K loop of one task through an NS-stage ring: `load(st, k0)` fills ring slot st with the
// tiles at K offset k0, `step(st)` consumes slot st. Every iteration commits one group (possibly
// empty), so wait_group<NS-2> always means "the group of this iteration's stage has landed".
template <int NS, typename Load, typename Step>
__device__ __forceinline__ void k_loop(int kb, int ke, Load &&load, Step &&step) {
  const int nk = ke - kb;
#pragma unroll
  for (int st = 0; st < NS - 1; ++st) {
    if (st < nk) load(st, (int64_t)(kb + st) * BK);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<NS - 2>();
    __syncthreads();  // stage kt visible to all; every warp is done with stage kt-1's slot
    const int nxt = kt + NS - 1;
    // this stage's DMMA first, then the refill of the slot read in the previous iteration: the
    // copies are issued while the DMMA execute
    step(kt % NS);
    if (nxt < nk) load(nxt % NS, (int64_t)(kb + nxt) * BK);
    cp_async_commit();
  }
  cp_async_wait<0>();
  __syncthreads();  // the ring may be refilled by the next task
}

// Split-K: store this piece's values (q-major: value q of every thread, so warps store
// contiguous runs), count the arrival; the last piece of the tile reads all partials in piece
// order and returns true with their sum in v. Unsplit tiles return true with v unchanged.
template <int NV, int NT>
__device__ __forceinline__ bool splitk_reduce(const PTask &t, double (&v)[NV], double *part, int *pcnt,
                                              int *ticket) {
  if (t.nsplit <= 1) return true;
  const int tid = threadIdx.x;
  double *mine = part + (int64_t)(t.pbase + t.sid) * (NV * NT);
#pragma unroll
  for (int q = 0; q < NV; ++q) __stcg(&mine[q * NT + tid], v[q]);
  __threadfence();
  __syncthreads();
  if (tid == 0) *ticket = atomicAdd(&pcnt[t.slot], 1);
  __syncthreads();
  const bool last = *ticket == t.nsplit - 1;
  __syncthreads();  // ticket is rewritten by the next task
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = 0.0;
  for (int sp = 0; sp < t.nsplit; ++sp) {  // piece order: deterministic sum
    const double *src = part + (int64_t)(t.pbase + sp) * (NV * NT);
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] += __ldcg(&src[q * NT + tid]);
  }
  if (tid == 0) pcnt[t.slot] = 0;  // every piece has arrived: the counter is free for the next launch
  return true;
}

__global__ void __launch_bounds__(kRealThreads, 2)
    gemm_f64_kernel(const GBlock *__restrict__ blocks, const PTask *__restrict__ tasks, int ntasks,
                    double *__restrict__ C, const double *__restrict__ A, const double *__restrict__ B,
                    double alpha, double beta, double *__restrict__ part, int *__restrict__ pcnt, int base_ok) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemR &s = *reinterpret_cast<SmemR *>(smem_raw);
  __shared__ int ticket;
  PL_STAMP(0);
  pdl_wait();  // operands, output and the split-K counters belong to earlier kernels too
  pdl_trigger();
  PL_STAMP(1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  [[maybe_unused]] int ntask = 0;
  for (int ti = blockIdx.x; ti < ntasks; ti += gridDim.x, ++ntask) {
    const PTask task = tasks[ti];
    const GBlock b = blocks[task.block];
    const int64_t m0 = task.m0, n0 = task.n0;
    const int vec = vec_flags(b, base_ok);
    // two accumulator sets, one per K sub-step of 8 in a stage (the 16 DMMA of a stage are
    // independent); their sum is (sub-step 0) + (sub-step 8)
    double acc[32], acc2[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = acc2[q] = 0.0;
    if (task.kind == 0 && task.ke > task.kb) {
      k_loop<NST>(task.kb, task.ke,
             [&](int st, int64_t k0) { load_tiles_r(s, st, b, A, B, m0, n0, k0, vec); },
             [&](int st) {
               // the warp's 32×32 as 2 × 4 blocks of 16×8 (m16n8k8), K in steps of 8
#pragma unroll
               for (int kk = 0; kk < BK; kk += 8) {
                 double *ac = kk == 0 ? acc : acc2;
                 double af[2][4], bf[4][2];
#pragma unroll
                 for (int mi = 0; mi < 2; ++mi) {
                   const int r = wm * 32 + mi * 16 + g;
                   af[mi][0] = s.A[st][kk + t][r];
                   af[mi][1] = s.A[st][kk + t][r + 8];
                   af[mi][2] = s.A[st][kk + t + 4][r];
                   af[mi][3] = s.A[st][kk + t + 4][r + 8];
                 }
#pragma unroll
                 for (int ni = 0; ni < 4; ++ni) {
                   bf[ni][0] = s.B[st][wn * 32 + ni * 8 + g][kk + t];
                   bf[ni][1] = s.B[st][wn * 32 + ni * 8 + g][kk + t + 4];
                 }
#pragma unroll
                 for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                   for (int ni = 0; ni < 4; ++ni)
                     dmma16(*reinterpret_cast<double(*)[4]>(&ac[(mi * 4 + ni) * 4]), af[mi], bf[ni]);
               }
             });
#pragma unroll
      for (int q = 0; q < 32; ++q) acc[q] += acc2[q];
    }
    if (ntask == 0) PL_STAMP(2);
    const bool fin = splitk_reduce<32, kRealThreads>(task, acc, part, pcnt, &ticket);
    if (ntask == 0) {
      PL_STAMP(3);
      PL_SET(6, 2ull * task.nsplit + (fin ? 1 : 0));
    }
    if (!fin) continue;
    // epilogue: C = α·acc + β·C, in four row groups of 8 (the old values of a group are loaded
    // before its first store). Row group R, value q (column block q/2, column 2t + q%2) is
    // acc[((R/2)·4 + q/2)·4 + (R%2)·2 + q%2] (the m16n8k8 fragments)
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int64_t i = m0 + wm * 32 + mi * 8 + g;
      double old[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int64_t j = n0 + wn * 32 + (q / 2) * 8 + 2 * t + (q % 2);
        old[q] = (beta != 0.0 && i < b.m && j < b.n) ? C[b.offC + i + j * b.ldc] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int64_t j = n0 + wn * 32 + (q / 2) * 8 + 2 * t + (q % 2);
        if (i < b.m && j < b.n) {
          double r = alpha * acc[((mi >> 1) * 4 + (q >> 1)) * 4 + (mi & 1) * 2 + (q & 1)];
          if (beta != 0.0) r = fma(beta, old[q], r);
          C[b.offC + i + j * b.ldc] = r;
        }
      }
    }
  }
  PL_SET(5, ntask);
  PL_STAMP(4);
}

// ---- complex ---------------------------------------------------------------------------
struct SmemC {
  double2 A[NST][BK][BM + CAPAD];  // op(A) tile, [k][row], whole complex elements
  double2 B[NST][BN][BK + CBPAD];  // op(B) tile, [col][k]
};

__device__ __forceinline__ void load_tiles_c(SmemC &s, int st, const GBlock &b, const double2 *A,
                                             const double2 *B, int64_t m0, int64_t n0, int64_t k0) {
  const int tid = threadIdx.x;
  if (b.opA == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BM * BK) / kCplxThreads; ++r) {
      const int e = tid + r * kCplxThreads;
      const int i = e % BM, l = e / BM;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      cp_async16(&s.A[st][l][i], A + b.offA + (ok ? gi + gl * b.lda : 0), ok ? 16 : 0);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BM * BK) / kCplxThreads; ++r) {
      const int e = tid + r * kCplxThreads;
      const int l = e % BK, i = e / BK;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      cp_async16(&s.A[st][l][i], A + b.offA + (ok ? gl + gi * b.lda : 0), ok ? 16 : 0);
    }
  }
  if (b.opB == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BN * BK) / kCplxThreads; ++r) {
      const int e = tid + r * kCplxThreads;
      const int l = e % BK, j = e / BK;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      cp_async16(&s.B[st][j][l], B + b.offB + (ok ? gl + gj * b.ldb : 0), ok ? 16 : 0);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BN * BK) / kCplxThreads; ++r) {
      const int e = tid + r * kCplxThreads;
      const int j = e % BN, l = e / BN;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      cp_async16(&s.B[st][j][l], B + b.offB + (ok ? gj + gl * b.ldb : 0), ok ? 16 : 0);
    }
  }
}

__global__ void __launch_bounds__(kCplxThreads, 2)
    gemm_c128_kernel(const GBlock *__restrict__ blocks, const PTask *__restrict__ tasks, int ntasks,
                     double2 *__restrict__ C, const double2 *__restrict__ A, const double2 *__restrict__ B,
                     CDbl alpha, CDbl beta, double *__restrict__ part, int *__restrict__ pcnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemC &s = *reinterpret_cast<SmemC *>(smem_raw);
  __shared__ int ticket;
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;  // 8 warps: 2 (m) x 4 (n)
  const int wm = warp & 1, wn = warp >> 1;                      // warp tile 32 x 16
  const int g = lane >> 2, t = lane & 3;
  const bool bz = beta.x == 0.0 && beta.y == 0.0;
  for (int ti = blockIdx.x; ti < ntasks; ti += gridDim.x) {
    const PTask task = tasks[ti];
    const GBlock b = blocks[task.block];
    // conjugation of an operand flips the sign of its imaginary part
    const double sa = (b.opA == TKB_OP_C) ? -1.0 : 1.0;
    const double sb = (b.opB == TKB_OP_C) ? -1.0 : 1.0;
    const int64_t m0 = task.m0, n0 = task.n0;
    // acc[(mi*2 + ni)*4 + {0,1}] = Re (columns 2t, 2t+1), +{2,3} = Im
    double acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.0;
    if (task.kind == 0 && task.ke > task.kb) {
      k_loop<NST>(task.kb, task.ke, [&](int st, int64_t k0) { load_tiles_c(s, st, b, A, B, m0, n0, k0); },
             [&](int st) {
#pragma unroll
               for (int kk = 0; kk < BK; kk += 4) {
                 double fr[4], fi[4], fin[4], gr[2], gi[2];
#pragma unroll
                 for (int mi = 0; mi < 4; ++mi) {
                   const double2 v = s.A[st][kk + t][wm * 32 + mi * 8 + g];
                   fr[mi] = v.x;
                   fi[mi] = sa * v.y;
                   fin[mi] = -fi[mi];
                 }
#pragma unroll
                 for (int ni = 0; ni < 2; ++ni) {
                   const double2 v = s.B[st][wn * 16 + ni * 8 + g][kk + t];
                   gr[ni] = v.x;
                   gi[ni] = sb * v.y;
                 }
#pragma unroll
                 for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                   for (int ni = 0; ni < 2; ++ni) {
                     double *a = &acc[(mi * 2 + ni) * 4];
                     dmma(a[0], a[1], fr[mi], gr[ni]);
                     dmma(a[0], a[1], fin[mi], gi[ni]);
                     dmma(a[2], a[3], fr[mi], gi[ni]);
                     dmma(a[2], a[3], fi[mi], gr[ni]);
                   }
               }
             });
    }
    if (!splitk_reduce<32, kCplxThreads>(task, acc, part, pcnt, &ticket)) continue;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int64_t i = m0 + wm * 32 + mi * 8 + g;
      if (i >= b.m) continue;
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t j = n0 + wn * 16 + ni * 8 + 2 * t + h;
          if (j >= b.n) continue;
          double2 *p = C + b.offC + i + j * b.ldc;
          const double vr = acc[(mi * 2 + ni) * 4 + h], vi = acc[(mi * 2 + ni) * 4 + 2 + h];
          double rr = alpha.x * vr - alpha.y * vi;
          double ri = alpha.x * vi + alpha.y * vr;
          if (!bz) {
            const double2 o = *p;
            rr = fma(beta.x, o.x, fma(-beta.y, o.y, rr));
            ri = fma(beta.x, o.y, fma(beta.y, o.x, ri));
          }
          *p = make_double2(rr, ri);
        }
      }
    }
  }
}

// ---- skinny blocks (n, k ≤ 16): one thread per output row, op(B) in shared memory -----------
// Such blocks (tall-skinny GEMMs against small MPO bonds) are bound by reading op(A) and
// writing C; the row kernel streams both exactly once with coalesced accesses for op N.
template <typename T>
__device__ __forceinline__ T ldA(const T *p, bool conj);
template <>
__device__ __forceinline__ double ldA<double>(const double *p, bool) { return __ldg(p); }
template <>
__device__ __forceinline__ double2 ldA<double2>(const double2 *p, bool conj) {
  double2 v = __ldg(p);
  if (conj) v.y = -v.y;
  return v;
}
__device__ __forceinline__ double mac(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ double2 mac(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
template <typename T>
__device__ __forceinline__ T make_beta(CDbl b);
template <>
__device__ __forceinline__ double make_beta<double>(CDbl b) { return b.x; }
template <>
__device__ __forceinline__ double2 make_beta<double2>(CDbl b) { return make_double2(b.x, b.y); }
__device__ __forceinline__ double zero(double) { return 0.0; }
__device__ __forceinline__ double2 zero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double scl(double v, CDbl a) { return a.x * v; }
__device__ __forceinline__ double2 scl(double2 v, CDbl a) {
  return make_double2(a.x * v.x - a.y * v.y, a.x * v.y + a.y * v.x);
}

// D bounds n and k of every block of the launch (2, 4, 6, 8 or 16) and R rows are handled per
// thread and pass: the R·k loads of op(A) of a pass are all issued before any arithmetic, so a
// thread keeps up to R·k loads in flight (R·D ≈ 16 values in registers, half that for complex
// data). Rows of a task: kSkinnyTaskRows, in passes of kSkinnyRows·R. Per element the arithmetic
// is acc = β·c (or 0), then acc = fma(α·a_l, op(B)_lj, acc) for l = 0 … k−1; rows where a_l was
// not loaded (invalid rows, l ≥ k) hold zeros and are not stored.
// rows per thread and pass for a width class: ≈ 16 values of op(A) in registers (complex: 8)
template <typename T, int DK>
constexpr int kSkinnyRowsPerPass = sizeof(T) == 8 ? (DK <= 4 ? 4 : DK <= 8 ? 2 : 1) : (DK <= 2 ? 4 : DK <= 4 ? 2 : 1);

// One task's rows in passes of kSkinnyRows·RR (rows per thread RR): all RR·k loads of op(A) are
// issued first; blocks with n, k ≤ DK ≤ D (op(B) staged with leading dimension D)
template <typename T, bool BZ, int D, int DK, int RR>
__device__ __forceinline__ void skinny_passes(int64_t m0, int64_t m, int kk, int n, const T *__restrict__ pa0,
                                              int64_t sa_i, int64_t sa_l, bool conjA, T *__restrict__ pc0,
                                              int64_t ldc, const T *Bs, CDbl alpha, CDbl beta) {
  static_assert(kSkinnyTaskRows % (kSkinnyRows * RR) == 0, "a task is a whole number of passes");
  for (int p0 = 0; p0 < kSkinnyTaskRows; p0 += kSkinnyRows * RR) {
    int64_t row[RR];
    bool valid[RR];
    T a[RR][DK];
#pragma unroll
    for (int r = 0; r < RR; ++r) {
      row[r] = m0 + p0 + r * kSkinnyRows + threadIdx.x;
      valid[r] = row[r] < m;
    }
#pragma unroll
    for (int r = 0; r < RR; ++r)
#pragma unroll
      for (int l = 0; l < DK; ++l)
        a[r][l] = (valid[r] && l < kk) ? ldA<T>(pa0 + row[r] * sa_i + l * sa_l, conjA) : zero(T{});
    // α·a once per element of op(A); each op(B)_lj is read from shared memory once per pass
    // and used for the RR rows
#pragma unroll
    for (int r = 0; r < RR; ++r)
#pragma unroll
      for (int l = 0; l < DK; ++l) a[r][l] = scl(a[r][l], alpha);
#pragma unroll
    for (int j = 0; j < DK; ++j) {
      if (j < n) {
        T acc[RR];
#pragma unroll
        for (int r = 0; r < RR; ++r) {
          acc[r] = zero(T{});
          if constexpr (!BZ)
            if (valid[r]) acc[r] = mac(pc0[row[r] + (int64_t)j * ldc], make_beta<T>(beta), zero(T{}));
        }
#pragma unroll
        for (int l = 0; l < DK; ++l) {
          if (l < kk) {
            const T bl = Bs[l + j * D];
#pragma unroll
            for (int r = 0; r < RR; ++r) acc[r] = mac(a[r][l], bl, acc[r]);
          }
        }
#pragma unroll
        for (int r = 0; r < RR; ++r)
          if (valid[r]) pc0[row[r] + (int64_t)j * ldc] = acc[r];
      }
    }
  }
}

// resident CTAs asked of the register allocator: the real β = 0 passes of widths 2 and 6 fit
// 48 registers (5 CTAs per SM), the other widths up to 8 fit 80 (3 CTAs), width 16 fits 128
template <typename T, bool BZ, int D>
constexpr int kSkinnyMinCtas = (sizeof(T) == 8 && BZ && (D == 2 || D == 6)) ? 5 : D <= 8 ? 3 : 2;

template <typename T, bool BZ, int D, int R>
__global__ void __launch_bounds__(kSkinnyRows, kSkinnyMinCtas<T, BZ, D>)
    gemm_skinny_kernel(const GBlock *__restrict__ blocks, const GTile *__restrict__ tasks, int64_t ntasks,
                       T *__restrict__ C, const T *__restrict__ A, const T *__restrict__ B, CDbl alpha,
                       CDbl beta) {
  __shared__ T Bs[D * D];
  // a contiguous, even share of the tasks per CTA: consecutive tasks mostly share their block,
  // so op(B) is staged again only when the block changes
  const int64_t t_begin = (int64_t)blockIdx.x * ntasks / gridDim.x;
  const int64_t t_end = (int64_t)(blockIdx.x + 1) * ntasks / gridDim.x;
  pdl_wait();
  pdl_trigger();
  int staged = -1;  // block whose op(B) is in Bs
  for (int64_t ti = t_begin; ti < t_end; ++ti) {
    const GTile tk = tasks[ti];
    const GBlock &b = blocks[tk.block];
    const int n = (int)b.n, k = (int)b.k;
    const int64_t m = b.m;
    const int kk = tk.kind == 0 ? k : 0;
    const bool conjA = b.opA == TKB_OP_C;
    const int64_t sa_l = (b.opA == TKB_OP_N) ? b.lda : 1;
    const int64_t sa_i = (b.opA == TKB_OP_N) ? 1 : b.lda;
    const int64_t ldc = b.ldc;
    const T *pa0 = A + b.offA;
    T *pc0 = C + b.offC;
    if (tk.block != staged) {  // uniform over the CTA
      __syncthreads();
      // op(B)(l, j), zero outside k × n (the row loops below run over the full D × D)
      for (int e = threadIdx.x; e < D * D; e += blockDim.x) {
        const int l = e % D, j = e / D;
        const int64_t idx = (b.opB == TKB_OP_N) ? b.offB + l + (int64_t)j * b.ldb : b.offB + j + (int64_t)l * b.ldb;
        Bs[e] = (l < k && j < n && tk.kind == 0) ? ldA<T>(B + idx, b.opB == TKB_OP_C) : zero(T{});
      }
      __syncthreads();
      staged = tk.block;
    }
    // blocks narrower than the launch's width class run a narrower pass with more rows per
    // thread (uniform per task), so their threads also keep ≈ 16 loads in flight
    if (D > 2 && kk <= 2 && n <= 2)
      skinny_passes<T, BZ, D, 2, kSkinnyRowsPerPass<T, 2>>(tk.m0, m, kk, n, pa0, sa_i, sa_l, conjA, pc0, ldc, Bs,
                                                           alpha, beta);
    else if (D > 4 && kk <= 4 && n <= 4)
      skinny_passes<T, BZ, D, 4, kSkinnyRowsPerPass<T, 4>>(tk.m0, m, kk, n, pa0, sa_i, sa_l, conjA, pc0, ldc, Bs,
                                                           alpha, beta);
    else
      skinny_passes<T, BZ, D, D, R>(tk.m0, m, kk, n, pa0, sa_i, sa_l, conjA, pc0, ldc, Bs, alpha, beta);
  }
}

}  // namespace

namespace {

template <typename T, bool BZ, int D>
int skinny_launch_t(tkb_ctx *ctx, const tkb_plan *p, T *C, const T *A, const T *B, CDbl a, CDbl bb) {
  auto k = gemm_skinny_kernel<T, BZ, D, kSkinnyRowsPerPass<T, D>>;
  const int per_sm = tkb_occupancy(ctx->device, (const void *)k, kSkinnyRows, 0);
  if (per_sm <= 0) return tkb_set_error(ctx, TKB_ERR_CUDA, "skinny GEMM: occupancy query failed");
  const int grid = (int)std::min<int64_t>(p->nsk, (int64_t)ctx->num_sms * per_sm);
  TKB_CUDA_TRY(ctx, launch_pdl(k, dim3(grid), dim3(kSkinnyRows), 0, ctx->stream, p->blocks, p->sktasks, p->nsk, C,
                               A, B, a, bb));
  return TKB_OK;
}

template <typename T, bool BZ>
int skinny_launch_d(tkb_ctx *ctx, const tkb_plan *p, T *C, const T *A, const T *B, CDbl a, CDbl bb) {
  const int d = p->sk_dim;
  if (d <= 2) return skinny_launch_t<T, BZ, 2>(ctx, p, C, A, B, a, bb);
  if (d <= 4) return skinny_launch_t<T, BZ, 4>(ctx, p, C, A, B, a, bb);
  if (d <= 6) return skinny_launch_t<T, BZ, 6>(ctx, p, C, A, B, a, bb);
  if (d <= 8) return skinny_launch_t<T, BZ, 8>(ctx, p, C, A, B, a, bb);
  return skinny_launch_t<T, BZ, 16>(ctx, p, C, A, B, a, bb);
}

}  // namespace

int tkb_gemm_skinny_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A,
                           const void *B, tkb_scalar alpha, tkb_scalar beta) {
  if (p->nsk == 0) return TKB_OK;
  const CDbl a{alpha.re, alpha.im}, bb{beta.re, beta.im};
  const bool bz = beta.re == 0.0 && beta.im == 0.0;
  int rc;
  if (p->dtype == TKB_F64)
    rc = bz ? skinny_launch_d<double, true>(ctx, p, (double *)C, (const double *)A, (const double *)B, a, bb)
            : skinny_launch_d<double, false>(ctx, p, (double *)C, (const double *)A, (const double *)B, a, bb);
  else
    rc = bz ? skinny_launch_d<double2, true>(ctx, p, (double2 *)C, (const double2 *)A, (const double2 *)B, a, bb)
            : skinny_launch_d<double2, false>(ctx, p, (double2 *)C, (const double2 *)A, (const double2 *)B, a, bb);
  if (rc != TKB_OK) return rc;
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

int tkb_gemm_plain_prepare(tkb_ctx *ctx, tkb_plan *p, const std::vector<GTile> &tiles) {
  const bool cplx = p->dtype == TKB_C128;
  const void *kfn = cplx ? (const void *)gemm_c128_kernel : (const void *)gemm_f64_kernel;
  const int threads = cplx ? kCplxThreads : kRealThreads;
  const size_t smem = cplx ? sizeof(SmemC) : sizeof(SmemR);
  const int per_sm = tkb_occupancy(ctx->device, kfn, threads, smem);
  if (per_sm <= 0) return tkb_set_error(ctx, TKB_ERR_CUDA, "plain GEMM: occupancy query failed");
  const int64_t slots = (int64_t)ctx->num_sms * per_sm;
  const int64_t nt = (int64_t)tiles.size();
  int64_t total = 0, maxnk = 1;
  std::vector<int64_t> nks(nt);
  for (int64_t i = 0; i < nt; ++i) {
    const GTile &t = tiles[i];
    nks[i] = t.kind == 0 ? (p->hblocks[t.block].k + BK - 1) / BK : 0;
    total += nks[i];
    maxnk = std::max(maxnk, nks[i]);
  }
  auto pieces = [&](int64_t nk, int64_t target) {
    return (int)std::min<int64_t>(p->max_pieces, std::max<int64_t>(1, (nk + target - 1) / target));
  };
  // the shortest piece length (at least min_piece_steps) whose tasks still fit the resident slots
  int64_t target = maxnk;
  if (nt < slots) {
    target = std::max<int64_t>(p->min_piece_steps, (total + slots - 1) / slots);
    for (; target < maxnk; ++target) {
      int64_t cnt = 0;
      for (int64_t i = 0; i < nt; ++i) cnt += pieces(nks[i], target);
      if (cnt <= slots) break;
    }
  }
  std::vector<PTask> tasks;
  int nslots = 0, npart = 0;
  for (int64_t i = 0; i < nt; ++i) {
    const GTile &t = tiles[i];
    const int nk = (int)nks[i];
    const int ks = t.kind == 0 ? pieces(nk, target) : 1;
    if (ks == 1) {
      tasks.push_back({t.block, t.m0, t.n0, t.kind, 0, nk, -1, 1, 0, 0});
    } else {
      const int slot = nslots++;
      for (int s = 0; s < ks; ++s)
        tasks.push_back({t.block, t.m0, t.n0, t.kind, s * nk / ks, (s + 1) * nk / ks, slot, ks, s, npart});
      npart += ks;
    }
  }
  // longest first; CTA b takes tasks b, b + grid, ... (a static cost-ordered queue)
  std::stable_sort(tasks.begin(), tasks.end(),
                   [](const PTask &x, const PTask &y) { return (x.ke - x.kb) > (y.ke - y.kb); });
  p->nptasks = (int64_t)tasks.size();
  p->pgrid = (int)std::min<int64_t>(p->nptasks, slots);
  cudaError_t e = cudaSuccess;
  if (!tasks.empty()) {
    e = cudaMalloc(&p->ptasks, tasks.size() * sizeof(PTask));
    if (e == cudaSuccess) e = cudaMemcpy(p->ptasks, tasks.data(), tasks.size() * sizeof(PTask), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && nslots > 0) {
    e = cudaMalloc((void **)&p->part, (size_t)npart * BM * BN * (cplx ? 2 : 1) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->pcnt, nslots * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->pcnt, 0, nslots * sizeof(int));
  }
  if (e != cudaSuccess)
    return tkb_set_error(ctx, TKB_ERR_CUDA, std::string("plain plan upload: ") + cudaGetErrorString(e));
  return TKB_OK;
}

int tkb_gemm_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B,
                    tkb_scalar alpha, tkb_scalar beta) {
  if (p->nptasks == 0) return TKB_OK;
  if (p->dtype == TKB_F64) {
    if (alpha.im != 0.0 || beta.im != 0.0)
      return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
    const size_t smem = sizeof(SmemR);
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(gemm_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int base_ok = (((uintptr_t)A & 15) == 0 ? 1 : 0) | (((uintptr_t)B & 15) == 0 ? 2 : 0);
    TKB_CUDA_TRY(ctx, launch_pdl(gemm_f64_kernel, dim3(p->pgrid), dim3(kRealThreads), smem, ctx->stream, p->blocks,
                                 (const PTask *)p->ptasks, (int)p->nptasks, (double *)C, (const double *)A,
                                 (const double *)B, alpha.re, beta.re, p->part, p->pcnt, base_ok));
  } else {
    if ((((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15) != 0)
      return tkb_set_error(ctx, TKB_ERR_ARG, "ComplexF64 data must be 16-byte aligned");
    const size_t smem = sizeof(SmemC);
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(gemm_c128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TKB_CUDA_TRY(ctx, launch_pdl(gemm_c128_kernel, dim3(p->pgrid), dim3(kCplxThreads), smem, ctx->stream, p->blocks,
                                 (const PTask *)p->ptasks, (int)p->nptasks, (double2 *)C, (const double2 *)A,
                                 (const double2 *)B, CDbl{alpha.re, alpha.im}, CDbl{beta.re, beta.im}, p->part,
                                 p->pcnt));
  }
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

#ifdef TKB_TIMELINE
// copies the plain kernel's per-CTA stamps out (kPlTlCtas × kPlTlSlots values) and clears them
extern "C" int tkb_timeline_read_plain(unsigned long long *out) {
  if (cudaMemcpyFromSymbol(out, tkb_tl_plain, sizeof(tkb_tl_plain)) != cudaSuccess) return -1;
  static unsigned long long zero[kPlTlCtas * kPlTlSlots];
  return cudaMemcpyToSymbol(tkb_tl_plain, zero, sizeof(tkb_tl_plain)) == cudaSuccess ? kPlTlSlots : -1;
}
#endif
