// Split-precision grouped block GEMM (Ozaki scheme I on the INT8 tensor pipe).
//
// Method (Ozaki, Ogita, Oishi & Rump 2012; Ootomo, Ozaki & Yokota 2024, "DGEMM on integer
// matrix multiplication unit"): every row i of op(A) is scaled by 2^-e_i (e_i the binary
// exponent bounding the row's largest magnitude) and cut into S int8 slices,
//     A_il·2^-e_i = Σ_{s=1..S} a^(s)_il · 2^-7s + r_il,   |a^(s)| ≤ 127,  |r| < 2^-7S,
// each slice being the truncated next 7 bits (the subtraction of the integer part is exact
// in FP64). Columns of op(B) are cut the same way with exponents f_j. Then
//     C_ij ≈ 2^(e_i+f_j) Σ_{d=2..S+1} 2^-7d P_d,ij ,   P_d = Σ_{s+t=d} a^(s) b^(t),
// where every P_d is an exact INT32 tensor-core accumulation (k·S·127² < 2^31). Terms with
// s+t > S+1 are below the truncation error and dropped. The recombination, the α/β update
// and everything after the integer products are FP64.
//
// ComplexF64 blocks are mapped to one real product: op(A) becomes the 2m×2k real matrix with
// row pairs (2r, 2r+1) = ([Re A_r, -Im A_r], [Im A_r, Re A_r]) and op(B) the 2k×n matrix
// [Re B; Im B], so rows 2r and 2r+1 of the real result are Re and Im of C_r.
//
// Slice layout in the workspace: per block, per slice, the rows of op(A) (op(B)ᵀ) are cut
// into panels of 128 (64) rows; a panel is a sequence of 32-byte K stages (one tensor-core
// K step), each stored as the canonical K-major "core matrix" layout of the tensor-core
// operand descriptors (8-row × 16-byte core matrices; 256 bytes between 8-row groups, 128
// bytes between the two 16-byte K chunks). One stage of one slice is therefore one
// contiguous 4 KiB (2 KiB) block that a single bulk copy moves into shared memory.
//
// Launches: exponent pass + slice pass (warp tasks of 32 rows × 64 K) + product pass:
//   tcgen05 kernel (default): one CTA per 128×64 output tile (and K range, when the K loop
//   is split across CTAs); one thread streams the S slice stages of A and B with
//   cp.async.bulk into a four-stage shared-memory ring and issues tcgen05.mma.kind::i8
//   (M=128, N=64, K=32) into S int32 accumulators held in tensor memory (S·64 of 512
//   columns); four warps read the accumulators back with tcgen05.ld and recombine them in
//   FP64.
//   mma.sync kernel (TKB_SPLIT_KERNEL=mma): the same products with int8 mma.sync.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "tkb_internal.h"

namespace {

constexpr int PANEL_A = 128, PANEL_B = 64;   // rows per panel
constexpr int KSTAGE = 32;                   // bytes of K per stage (one tensor-core K step)
constexpr int NSTAGE = 4;                    // depth of the shared-memory ring
constexpr int SMAX = 7;

struct SliceJob {
  int32_t block;
  int32_t operand;  // 0 = rows of op(A), 1 = columns of op(B)
};

struct CDbl {
  double x, y;
};

// byte offset of (row r, K byte kb) inside one slice plane
__host__ __device__ __forceinline__ int64_t slice_off(int64_t r, int64_t kb, int64_t kpad, int pr) {
  const int64_t panel = r / pr, rr = r % pr;
  const int64_t stg = kb >> 5, kk = kb & 31;
  return panel * (pr * kpad) + stg * (pr * KSTAGE) + (rr >> 3) * 256 + (kk >> 4) * 128 +
         (rr & 7) * 16 + (kk & 15);
}

// element (r, l) of the logical real operand (rows r of M' or N', column l of K')
__device__ __forceinline__ double op_elem(const GBlock &b, int operand, int cplx,
                                          const double *X, int64_t r, int64_t l) {
  if (operand == 0) {
    if (!cplx) {
      const int64_t idx = (b.opA == TKB_OP_N) ? b.offA + r + l * b.lda : b.offA + l + r * b.lda;
      return X[idx];
    }
    const int64_t rr = r >> 1;
    const bool odd = r & 1;
    const bool second = l >= b.k;
    const int64_t ll = second ? l - b.k : l;
    const int64_t idx = (b.opA == TKB_OP_N) ? b.offA + rr + ll * b.lda : b.offA + ll + rr * b.lda;
    const double re = X[2 * idx];
    double im = X[2 * idx + 1];
    if (b.opA == TKB_OP_C) im = -im;
    if (!odd) return second ? -im : re;  // row 2r:   [Re, -Im]
    return second ? re : im;             // row 2r+1: [Im,  Re]
  }
  if (!cplx) {
    const int64_t idx = (b.opB == TKB_OP_N) ? b.offB + l + r * b.ldb : b.offB + r + l * b.ldb;
    return X[idx];
  }
  const bool second = l >= b.k;
  const int64_t ll = second ? l - b.k : l;
  const int64_t idx = (b.opB == TKB_OP_N) ? b.offB + ll + r * b.ldb : b.offB + r + ll * b.ldb;
  if (!second) return X[2 * idx];
  const double im = X[2 * idx + 1];
  return (b.opB == TKB_OP_C) ? -im : im;
}

// Slicing of the operands, in two launches over fine-grained warp tasks. A task is one
// group of 32 operand rows × one chunk of 128 K positions (rows of all jobs enumerated
// through the task prefix sums; padding rows and padding K included, so the padded
// slices are written as zeros).
//   expo_kernel : per task the partial row maxima, folded into the row exponents with an
//                 integer atomicMax (the exponent array starts at a very negative value,
//                 byte 0x80 everywhere); complex row pairs fold into both rows.
//   slice_kernel: per task the S slices of every element, packed into 16-byte (row-
//                 contiguous operands, lane = row) or 4-byte (lane = 4 consecutive K)
//                 stores in the tensor-core operand layout.
// Row-contiguous operands are real op(A) = A and real op(B) = Bᵀ (consecutive rows are
// consecutive addresses); the others read 4 consecutive K positions per lane.
constexpr int KCHUNK = 64;

struct TaskLoc {
  SliceJob job;
  int64_t r0, l0;
};

__device__ __forceinline__ TaskLoc locate_task(int64_t t, const int64_t *__restrict__ task_begin,
                                               const SliceJob *__restrict__ jobs, int njobs,
                                               const GBlock *__restrict__ blocks) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (task_begin[mid] <= t) lo = mid; else hi = mid - 1;
  }
  const SliceJob job = jobs[lo];
  const GBlock &b = blocks[job.block];
  const int64_t nkc = (b.kpad + KCHUNK - 1) / KCHUNK;
  const int64_t rel = t - task_begin[lo];
  return TaskLoc{job, (rel / nkc) * 32, (rel % nkc) * KCHUNK};
}

__device__ __forceinline__ bool row_contiguous(const GBlock &b, int op, int cplx) {
  return !cplx && ((op == 0 && b.opA == TKB_OP_N) || (op == 1 && b.opB != TKB_OP_N));
}

__global__ void __launch_bounds__(256)
    expo_kernel(const GBlock *__restrict__ blocks, const int64_t *__restrict__ task_begin,
                const SliceJob *__restrict__ jobs, int njobs, int64_t ntasks, int cplx,
                const double *__restrict__ A, const double *__restrict__ B, int8_t *ws) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntasks; t += nw) {
    const TaskLoc L = locate_task(t, task_begin, jobs, njobs, blocks);
    const GBlock &b = blocks[L.job.block];
    const int op = L.job.operand;
    const int64_t Mlog = op == 0 ? (cplx ? 2 * b.m : b.m) : b.n;
    const int64_t Klog = cplx ? 2 * b.k : b.k;
    int32_t *expo = reinterpret_cast<int32_t *>(ws + (op == 0 ? b.wsEA : b.wsEB));
    const double *X = op == 0 ? A : B;
    const int64_t l1 = min(L.l0 + KCHUNK, Klog);
    if (row_contiguous(b, op, cplx)) {
      const int64_t xo = op == 0 ? b.offA : b.offB;
      const int64_t ld = op == 0 ? b.lda : b.ldb;
      const int64_t r = L.r0 + lane;
      if (r >= Mlog || L.l0 >= l1) continue;
      double mx = 0.0;
      for (int64_t c = L.l0; c < l1; c += 16) {
        double v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = (c + q < l1) ? X[xo + r + (c + q) * ld] : 0.0;
#pragma unroll
        for (int q = 0; q < 16; ++q) mx = fmax(mx, fabs(v[q]));
      }
      if (mx > 0.0) {
        int e;
        frexp(mx, &e);
        atomicMax(&expo[r], e);
      }
      continue;
    }
    // lane = 2 consecutive K positions; 8 rows per batch so 16 loads are in flight per lane
    for (int rb = 0; rb < 32; rb += 8) {
      double mx[8];
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int64_t r = L.r0 + rb + rr;
        mx[rr] = 0.0;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int64_t l = L.l0 + 2 * lane + q;
          if (r < Mlog && l < l1) mx[rr] = fmax(mx[rr], fabs(op_elem(b, op, cplx, X, r, l)));
        }
      }
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int64_t r = L.r0 + rb + rr;
        double m = mx[rr];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0 && r < Mlog && m > 0.0) {
          int e;
          frexp(m, &e);
          atomicMax(&expo[r], e);
          if (cplx && op == 0) atomicMax(&expo[r ^ 1], e);  // a complex row pair shares one exponent
        }
      }
    }
  }
}

template <int S>
__device__ __forceinline__ void cut(double x, uint32_t (&w)[S], int shift) {
#pragma unroll
  for (int s = 0; s < S; ++s) {
    x *= 128.0;
    const double qd = trunc(x);
    x -= qd;
    w[s] |= ((uint32_t)(uint8_t)(int8_t)qd) << shift;
  }
}

template <int S>
__global__ void __launch_bounds__(256)
    slice_kernel(const GBlock *__restrict__ blocks, const int64_t *__restrict__ task_begin,
                 const SliceJob *__restrict__ jobs, int njobs, int64_t ntasks, int cplx,
                 const double *__restrict__ A, const double *__restrict__ B, int8_t *ws) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntasks; t += nw) {
    const TaskLoc L = locate_task(t, task_begin, jobs, njobs, blocks);
    const GBlock &b = blocks[L.job.block];
    const int op = L.job.operand;
    const int64_t Mlog = op == 0 ? (cplx ? 2 * b.m : b.m) : b.n;
    const int64_t Klog = cplx ? 2 * b.k : b.k;
    const int64_t rows_pad = op == 0 ? b.mpad : b.npad;
    const int pr = op == 0 ? PANEL_A : PANEL_B;
    const int64_t kpad = b.kpad;
    int8_t *base = ws + (op == 0 ? b.wsA : b.wsB);
    const int32_t *expo = reinterpret_cast<const int32_t *>(ws + (op == 0 ? b.wsEA : b.wsEB));
    const double *X = op == 0 ? A : B;
    const int64_t plane = rows_pad * kpad;
    const int64_t l1 = min(L.l0 + KCHUNK, kpad);
    if (row_contiguous(b, op, cplx)) {
      const int64_t xo = op == 0 ? b.offA : b.offB;
      const int64_t ld = op == 0 ? b.lda : b.ldb;
      const int64_t r = L.r0 + lane;
      const bool valid = r < Mlog;
      const int e = valid ? max(expo[r], -1100) : 0;
      for (int64_t c = L.l0; c < l1; c += 16) {
        uint32_t w[4][S];
#pragma unroll
        for (int h = 0; h < 4; ++h)
#pragma unroll
          for (int s = 0; s < S; ++s) w[h][s] = 0u;
        double v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = (valid && c + q < Klog) ? X[xo + r + (c + q) * ld] : 0.0;
#pragma unroll
        for (int q = 0; q < 16; ++q) cut<S>(ldexp(v[q], -e), w[q >> 2], 8 * (q & 3));
        const int64_t off = slice_off(r, c, kpad, pr);
#pragma unroll
        for (int s = 0; s < S; ++s)
          *reinterpret_cast<uint4 *>(base + s * plane + off) = make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
      }
      continue;
    }
    // lane = 2 consecutive K positions (64 per warp); 8 rows per batch, loads first
    const int64_t lb = L.l0 + 2 * lane;
    for (int rb = 0; rb < 32; rb += 8) {
      double v[8][2];
      int ex[8];
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int64_t r = L.r0 + rb + rr;
        const bool valid = r < Mlog;
        ex[rr] = valid ? max(expo[r], -1100) : 0;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int64_t l = lb + q;
          v[rr][q] = (valid && l < Klog) ? op_elem(b, op, cplx, X, r, l) : 0.0;
        }
      }
      if (lb >= l1) continue;
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int64_t r = L.r0 + rb + rr;
        uint32_t w[S];
#pragma unroll
        for (int s = 0; s < S; ++s) w[s] = 0u;
#pragma unroll
        for (int q = 0; q < 2; ++q) cut<S>(ldexp(v[rr][q], -ex[rr]), w, 8 * q);
        const int64_t off = slice_off(r, lb, kpad, pr);
#pragma unroll
        for (int s = 0; s < S; ++s) *reinterpret_cast<uint16_t *>(base + s * plane + off) = (uint16_t)w[s];
      }
    }
  }
}

// ---- shared epilogue: recombine one output value --------------------------------------------
__device__ __forceinline__ void store_out(double v, int64_t i, int64_t j, const GBlock &b, int cplx,
                                          double *C, CDbl alpha, CDbl beta, bool bz, int lane_xor) {
  const int64_t Mreal = cplx ? 2 * b.m : b.m;
  if (!cplx) {
    if (i < b.m && j < b.n) {
      double *p = C + b.offC + i + j * b.ldc;
      double r = alpha.x * v;
      if (!bz) r = fma(beta.x, *p, r);
      *p = r;
    }
    return;
  }
  const double w = __shfl_xor_sync(0xffffffffu, v, lane_xor);  // partner row i ^ 1
  if (!(i & 1) && i < Mreal && j < b.n) {
    double2 *p = reinterpret_cast<double2 *>(C) + b.offC + (i >> 1) + j * b.ldc;
    double rr = alpha.x * v - alpha.y * w;
    double ri = alpha.x * w + alpha.y * v;
    if (!bz) {
      const double2 o = *p;
      rr = fma(beta.x, o.x, fma(-beta.y, o.y, rr));
      ri = fma(beta.x, o.y, fma(beta.y, o.x, ri));
    }
    *p = make_double2(rr, ri);
  }
}

// ---- tcgen05 product kernel --------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// bounded wait on a phase parity: false once 2 s of wall time have passed
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if (globaltimer_ns() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// K-major operand descriptor, no swizzle: 8-row × 16-byte core matrices, LBO between the
// two K core matrices of one instruction, SBO between 8-row groups; version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

constexpr uint32_t kTmemCols = 512;
// instruction descriptor: D s32 (bits 4-5 = 2), A/B signed int8 (bits 7-9, 10-12 = 1),
// both K-major, N = 64 (bits 17-22 = 64>>3), M = 128 (bits 24-28 = 128>>4)
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// One product task: output tile (m0, n0) of a block, K stages [kb, ke). When a tile's K
// range is split over nsplit CTAs (few tiles, long K), each CTA recombines its own int32
// diagonals into an FP64 partial tile and stores it (plain coalesced stores) in partial
// buffer pbase + sid; the CTA that arrives last on the tile's counter adds the partials in
// split order (deterministic), scales, writes C and resets the counter for the next launch.
struct SplitTile {
  int32_t block, m0, n0, kind;
  int32_t kb, ke, slot, nsplit;
  int32_t sid, pbase;
};

template <int S>
__global__ void __launch_bounds__(128, 1)
    gemm_split_tc_kernel(const GBlock *__restrict__ blocks, const SplitTile *__restrict__ tiles,
                         const int8_t *__restrict__ ws, int cplx, double *__restrict__ C, CDbl alpha,
                         CDbl beta, int *err, double *__restrict__ part, int *__restrict__ pcnt) {
  constexpr uint32_t A_BYTES = S * PANEL_A * KSTAGE, B_BYTES = S * PANEL_B * KSTAGE;
  constexpr uint32_t STAGE = A_BYTES + B_BYTES;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * STAGE);
  uint64_t *empty = full + NSTAGE;
  uint64_t *done = full + 2 * NSTAGE;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(full + 2 * NSTAGE + 1);
  int *ticket = reinterpret_cast<int *>(full + 2 * NSTAGE + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const SplitTile tile = tiles[blockIdx.x];
  const GBlock b = blocks[tile.block];
  const bool has_k = tile.kind == 0;
  const int kb = tile.kb;
  const int nk = has_k ? tile.ke - tile.kb : 0;
  const bool bz = beta.x == 0.0 && beta.y == 0.0;

  if (tid == 0) {
#pragma unroll
    for (int st = 0; st < NSTAGE; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0 && has_k) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = has_k ? *tmem_slot : 0u;

  if (has_k && tid == 0) {
    const int8_t *gA = ws + b.wsA + (int64_t)(tile.m0 / PANEL_A) * PANEL_A * b.kpad;
    const int8_t *gB = ws + b.wsB + (int64_t)(tile.n0 / PANEL_B) * PANEL_B * b.kpad;
    const int64_t planeA = (int64_t)b.mpad * b.kpad, planeB = (int64_t)b.npad * b.kpad;
    auto load = [&](int kt, int st) {  // kt: local stage index, global stage kb + kt
      unsigned char *sa = smem + st * STAGE;
      const int64_t kg = kb + kt;
      mbar_expect_tx(&full[st], STAGE);
#pragma unroll
      for (int s = 0; s < S; ++s)
        bulk_g2s(sa + s * (PANEL_A * KSTAGE), gA + s * planeA + kg * PANEL_A * KSTAGE,
                 PANEL_A * KSTAGE, &full[st]);
#pragma unroll
      for (int s = 0; s < S; ++s)
        bulk_g2s(sa + A_BYTES + s * (PANEL_B * KSTAGE), gB + s * planeB + kg * PANEL_B * KSTAGE,
                 PANEL_B * KSTAGE, &full[st]);
    };
    // NSTAGE-deep ring: stage kt lives in slot kt % NSTAGE; its n-th use has parity n & 1.
    // After issuing the products of stage kt, the slot of stage kt-1 is refilled with stage
    // kt-1+NSTAGE once those older products have drained (their commit on empty[]), so the
    // tensor pipe always has the current stage queued while the copy engine refills.
    bool ok = true;
    int issued = 0, consumed = 0;  // stages loaded / waited on
    for (; issued < nk && issued < NSTAGE; ++issued) load(issued, issued);
    // descriptor templates: only the start address changes between stages
    const uint32_t ring0 = smem_u32(smem);
    for (int kt = 0; kt < nk && ok; ++kt) {
      const int st = kt % NSTAGE;
      ok = mbar_wait(&full[st], (kt / NSTAGE) & 1);
      if (!ok) break;
      ++consumed;
      tc_fence_after();
      const uint32_t a0 = ring0 + st * STAGE, b0 = a0 + A_BYTES;
      uint64_t ad[S], bd[S];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        ad[s] = umma_desc(a0 + s * (PANEL_A * KSTAGE), 128, 256);
        bd[s] = umma_desc(b0 + s * (PANEL_B * KSTAGE), 128, 256);
      }
#pragma unroll
      for (int s = 0; s < S; ++s) {
#pragma unroll
        for (int t = 0; t < S - s; ++t)
          umma_i8(tmem + (uint32_t)((s + t) * 64), ad[s], bd[t], kIdescI8, (kt > 0 || s > 0) ? 1u : 0u);
      }
      umma_commit(&empty[st]);
      if (kt >= 1) {
        const int prev = kt - 1, ps = prev % NSTAGE, nxt = prev + NSTAGE;
        if (nxt < nk) {
          ok = mbar_wait(&empty[ps], (prev / NSTAGE) & 1);
          if (!ok) break;
          load(nxt, ps);
          ++issued;
        }
      }
    }
    umma_commit(done);
    if (!ok) {
      atomicExch(err, 1);
      // let every bulk copy still in flight land before the CTA can exit (bounded)
      for (int k = consumed; k < issued; ++k) mbar_wait(&full[k % NSTAGE], (k / NSTAGE) & 1);
    }
  }
  if (has_k) {
    if (!mbar_wait(done, 0)) atomicExch(err, 2);
    tc_fence_after();
  }
  __syncwarp();  // tcgen05.ld is warp-collective: reconverge after the divergent waits
  // epilogue: warp w owns accumulator rows 32w..32w+31 (TMEM lanes)
  const int32_t *eA = reinterpret_cast<const int32_t *>(ws + b.wsEA);
  const int32_t *eB = reinterpret_cast<const int32_t *>(ws + b.wsEB);
  const int64_t Mreal = cplx ? 2 * b.m : b.m;
  const int row = 32 * warp + lane;
  const int64_t i = tile.m0 + row;
  // exponents of all-zero rows stay at the 0x80808080 reset value: clamp before adding
  const int ei = (has_k && i < Mreal) ? max(eA[i], -1100) : 0;
  // this CTA's FP64 recombination of its diagonals: chunk c of 16 columns
  auto recombine = [&](int c, double (&v)[16]) {
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = 0.0;
    if (!has_k) return;
#pragma unroll
    for (int d = S - 1; d >= 0; --d) {
      uint32_t r[16];
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(d * 64 + c * 16), r);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] += ldexp((double)(int32_t)r[q], -7 * (d + 2));
    }
  };
  bool write_out = true;
  if (tile.nsplit > 1) {
    double *mine = part + (int64_t)(tile.pbase + tile.sid) * (64 * 128);  // [col][row]
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      double v[16];
      recombine(c, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) __stcg(&mine[(c * 16 + q) * 128 + row], v[q]);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) *ticket = atomicAdd(&pcnt[tile.slot], 1);
    __syncthreads();
    write_out = (*ticket == tile.nsplit - 1);
    if (write_out) __threadfence();
  }
  if (write_out) {
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      double v[16];
      if (tile.nsplit > 1) {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = 0.0;
        for (int sp = 0; sp < tile.nsplit; ++sp) {
          const double *src = part + (int64_t)(tile.pbase + sp) * (64 * 128);
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] += __ldcg(&src[(c * 16 + q) * 128 + row]);
        }
      } else {
        recombine(c, v);
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int64_t j = tile.n0 + c * 16 + q;
        double val = v[q];
        if (has_k) val = ldexp(val, ei + ((j < b.n) ? max(eB[j], -1100) : 0));
        store_out(val, i, j, b, cplx, C, alpha, beta, bz, 1);
      }
    }
    if (tile.nsplit > 1 && tid == 0) pcnt[tile.slot] = 0;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0 && has_k) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
  }
}

// ---- mma.sync product kernel (comparison path) -------------------------------------------------
constexpr int SBM = 64, SBN = 64, SBK = 32;
constexpr int SPITCH = 48;  // smem row pitch in bytes: conflict-free fragment loads

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

__device__ __forceinline__ void imma(int (&c)[4], const int (&a)[4], const int (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int S>
__device__ __forceinline__ void load_stage(int8_t *As, int8_t *Bs, const GBlock &b, const int8_t *ws,
                                           int64_t m0, int64_t n0, int64_t k0) {
  const int64_t planeA = (int64_t)b.mpad * b.kpad, planeB = (int64_t)b.npad * b.kpad;
  for (int c = threadIdx.x; c < 2 * S * 128; c += blockDim.x) {
    const int op = c / (S * 128);
    const int rem = c % (S * 128);
    const int s = rem / 128, q = rem % 128;
    const int row = q >> 1, half = q & 1;
    if (op == 0) {
      const int8_t *g = ws + b.wsA + s * planeA + slice_off(m0 + row, k0 + half * 16, b.kpad, PANEL_A);
      cp_async16(As + (s * SBM + row) * SPITCH + half * 16, g);
    } else {
      const int8_t *g = ws + b.wsB + s * planeB + slice_off(n0 + row, k0 + half * 16, b.kpad, PANEL_B);
      cp_async16(Bs + (s * SBN + row) * SPITCH + half * 16, g);
    }
  }
}

template <int S>
__global__ void __launch_bounds__(256)
    gemm_split_mma_kernel(const GBlock *__restrict__ blocks, const GTile *__restrict__ tiles,
                          int ntiles, int *counters, const int8_t *__restrict__ ws, int cplx,
                          double *__restrict__ C, CDbl alpha, CDbl beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int8_t *As0 = reinterpret_cast<int8_t *>(smem_raw);
  const int stage_bytes = 2 * S * SBM * SPITCH;
  __shared__ int next_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;  // 2 x 4 warps, warp tile 32 x 16
  const int g = lane >> 2, tig = lane & 3;
  const bool bz = beta.x == 0.0 && beta.y == 0.0;
  while (true) {
    if (threadIdx.x == 0) next_tile = atomicAdd(&counters[2], 1);
    __syncthreads();
    const int ti = next_tile;
    __syncthreads();
    if (ti >= ntiles) break;
    const GTile tile = tiles[ti];
    const GBlock b = blocks[tile.block];
    // mma.sync tiles are 64 x 64 quarters of the 128 x 64 tcgen05 tiles
    for (int half = 0; half < 2; ++half) {
      const int64_t m0 = tile.m0 + half * 64, n0 = tile.n0;
      int acc[S][2][2][4];
#pragma unroll
      for (int d = 0; d < S; ++d)
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[d][mt][nt][q] = 0;
      const int64_t nk = b.kpad / SBK;
      if (tile.kind == 0 && nk > 0) {
        load_stage<S>(As0, As0 + S * SBM * SPITCH, b, ws, m0, n0, 0);
        cp_commit();
        for (int64_t kt = 0; kt < nk; ++kt) {
          int8_t *As = As0 + (kt & 1) * stage_bytes;
          int8_t *Bs = As + S * SBM * SPITCH;
          if (kt + 1 < nk) {
            int8_t *An = As0 + ((kt + 1) & 1) * stage_bytes;
            load_stage<S>(An, An + S * SBM * SPITCH, b, ws, m0, n0, (kt + 1) * SBK);
            cp_commit();
            cp_wait1();
          } else {
            cp_wait0();
          }
          __syncthreads();
#pragma unroll
          for (int s = 0; s < S; ++s) {
            int af[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
              const int8_t *p = As + (s * SBM + wm * 32 + mt * 16 + g) * SPITCH + tig * 4;
              af[mt][0] = *reinterpret_cast<const int *>(p);
              af[mt][1] = *reinterpret_cast<const int *>(p + 8 * SPITCH);
              af[mt][2] = *reinterpret_cast<const int *>(p + 16);
              af[mt][3] = *reinterpret_cast<const int *>(p + 8 * SPITCH + 16);
            }
#pragma unroll
            for (int t = 0; t < S - s; ++t) {
              int bf[2][2];
#pragma unroll
              for (int nt = 0; nt < 2; ++nt) {
                const int8_t *p = Bs + (t * SBN + wn * 16 + nt * 8 + g) * SPITCH + tig * 4;
                bf[nt][0] = *reinterpret_cast<const int *>(p);
                bf[nt][1] = *reinterpret_cast<const int *>(p + 16);
              }
#pragma unroll
              for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) imma(acc[s + t][mt][nt], af[mt], bf[nt]);
            }
          }
          __syncthreads();
        }
      }
      const int32_t *eA = reinterpret_cast<const int32_t *>(ws + b.wsEA);
      const int32_t *eB = reinterpret_cast<const int32_t *>(ws + b.wsEB);
      const int64_t Mreal = cplx ? 2 * b.m : b.m;
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
          const int64_t i = m0 + wm * 32 + mt * 16 + g + hr * 8;
#pragma unroll
          for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int hc = 0; hc < 2; ++hc) {
              const int64_t j = n0 + wn * 16 + nt * 8 + 2 * tig + hc;
              double v = 0.0;
              if (tile.kind == 0) {
#pragma unroll
                for (int d = S - 1; d >= 0; --d) v += ldexp((double)acc[d][mt][nt][hr * 2 + hc], -7 * (d + 2));
                v = ldexp(v, ((i < Mreal) ? max(eA[i], -1100) : 0) + ((j < b.n) ? max(eB[j], -1100) : 0));
              }
              store_out(v, i, j, b, cplx, C, alpha, beta, bz, 4);
            }
        }
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const int done = atomicAdd(&counters[3], 1);
    if (done == (int)gridDim.x - 1) {
      atomicExch(&counters[2], 0);
      atomicExch(&counters[3], 0);
      __threadfence();
    }
  }
}

bool use_mma_sync() {
  const char *e = std::getenv("TKB_SPLIT_KERNEL");
  return e && std::strcmp(e, "mma") == 0;
}

template <int S>
int launch_split(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B, CDbl a, CDbl b) {
  const int cplx = p->dtype == TKB_C128 ? 1 : 0;
  if (p->nsrows > 0) {
    // one warp per (32-row group, 128-K chunk) task
    const int grid = (int)std::min<int64_t>((p->nsrows + 7) / 8, (int64_t)ctx->num_sms * 16);
    int8_t *ws = (int8_t *)ctx->ws;
    TKB_CUDA_TRY(ctx, cudaMemsetAsync(ws + p->expo_off, 0x80, p->expo_bytes, ctx->stream));
    expo_kernel<<<grid, 256, 0, ctx->stream>>>(p->blocks, p->srow_begin, (const SliceJob *)p->sjobs,
                                               p->nsjobs, p->nsrows, cplx, (const double *)A,
                                               (const double *)B, ws);
    slice_kernel<S><<<grid, 256, 0, ctx->stream>>>(p->blocks, p->srow_begin, (const SliceJob *)p->sjobs,
                                                   p->nsjobs, p->nsrows, cplx, (const double *)A,
                                                   (const double *)B, ws);
    ctx->launches += 2;
    TKB_CUDA_TRY(ctx, cudaGetLastError());
  }
  if (use_mma_sync()) {
    const size_t smem = 2 * (size_t)(2 * S * SBM * SPITCH);
    auto k = gemm_split_mma_kernel<S>;
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (int)std::min<int64_t>(p->nstiles, (int64_t)ctx->num_sms * 2);
    k<<<grid, 256, smem, ctx->stream>>>(p->blocks, p->stiles, (int)p->nstiles, ctx->counters,
                                        (const int8_t *)ctx->ws, cplx, (double *)C, a, b);
  } else {
    const size_t smem = NSTAGE * (size_t)S * (PANEL_A + PANEL_B) * KSTAGE + 128;
    auto k = gemm_split_tc_kernel<S>;
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<(int)p->nkstiles, 128, smem, ctx->stream>>>(p->blocks, (const SplitTile *)p->kstiles,
                                                    (const int8_t *)ctx->ws, cplx, (double *)C, a, b,
                                                    ctx->counters + 8, p->part, p->pcnt);
  }
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

int64_t roundup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

}  // namespace

int tkb_gemm_split_prepare(tkb_ctx *ctx, tkb_plan *p) {
  const bool cplx = p->dtype == TKB_C128;
  int S = p->slices;
  if (S <= 0) S = 7;
  if (S < 3 || S > SMAX) return tkb_set_error(ctx, TKB_ERR_UNSUPPORTED, "slices must be in 3..7");
  p->slices = S;
  size_t off = 0;
  std::vector<SliceJob> jobs;
  std::vector<int64_t> grp_begin;
  std::vector<GTile> tiles;
  int64_t ngroups = 0;
  for (size_t bi = 0; bi < p->hblocks.size(); ++bi) {
    GBlock &b = p->hblocks[bi];
    const int64_t M = cplx ? 2 * b.m : b.m;
    const int64_t K = cplx ? 2 * b.k : b.k;
    b.mpad = (int32_t)roundup(std::max<int64_t>(M, 1), PANEL_A);
    b.npad = (int32_t)roundup(std::max<int64_t>(b.n, 1), PANEL_B);
    b.kpad = (int32_t)roundup(std::max<int64_t>(K, 1), KSTAGE);
    if (b.m == 0 || b.n == 0 || b.skinny) continue;
    b.wsA = (int64_t)off;
    off += (size_t)S * b.mpad * b.kpad;
    b.wsB = (int64_t)off;
    off += (size_t)S * b.npad * b.kpad;
    off = roundup((int64_t)off, 256);
    const int kind = b.k > 0 ? 0 : 1;
    if (kind == 0) {
      const int64_t nkc = (b.kpad + KCHUNK - 1) / KCHUNK;  // K chunks (slicing tasks per row group)
      jobs.push_back({(int32_t)bi, 0});
      grp_begin.push_back(ngroups);
      ngroups += (b.mpad / 32) * nkc;
      jobs.push_back({(int32_t)bi, 1});
      grp_begin.push_back(ngroups);
      ngroups += (b.npad / 32) * nkc;
    }
    for (int64_t m0 = 0; m0 < M; m0 += PANEL_A)
      for (int64_t n0 = 0; n0 < b.n; n0 += PANEL_B) tiles.push_back({(int32_t)bi, (int32_t)m0, (int32_t)n0, kind});
  }
  // exponent arrays of every block in one contiguous region (reset to byte 0x80 per launch)
  p->expo_off = (int64_t)off;
  for (size_t bi = 0; bi < p->hblocks.size(); ++bi) {
    GBlock &b = p->hblocks[bi];
    if (b.m == 0 || b.n == 0 || b.skinny) continue;
    b.wsEA = (int64_t)off;
    off += (size_t)b.mpad * 4;
    b.wsEB = (int64_t)off;
    off += (size_t)b.npad * 4;
  }
  p->expo_bytes = (int64_t)off - p->expo_off;
  off = roundup((int64_t)off, 256);
  std::stable_sort(tiles.begin(), tiles.end(), [&](const GTile &x, const GTile &y) {
    return p->hblocks[x.block].kpad > p->hblocks[y.block].kpad;
  });
  // tcgen05 tasks: split the K range of tiles when there are too few tiles to occupy every
  // SM twice, keeping at least two K stages per task
  std::vector<SplitTile> kt;
  int nslots = 0, npart = 0;
  {
    const int64_t nt = (int64_t)tiles.size();
    int KS = 1;
    // one CTA per SM (shared-memory ring): keep every task in the first wave
    if (nt > 0 && nt < (int64_t)ctx->num_sms)
      KS = (int)std::min<int64_t>(8, (int64_t)ctx->num_sms / nt);
    for (const GTile &t : tiles) {
      const int nk = p->hblocks[t.block].kpad / KSTAGE;
      const int ks = t.kind == 0 ? std::max(1, std::min(KS, nk / 4)) : 1;  // ≥ 4 K stages per task
      if (ks == 1) {
        kt.push_back({t.block, t.m0, t.n0, t.kind, 0, nk, -1, 1, 0, 0});
      } else {
        const int slot = nslots++;
        for (int s = 0; s < ks; ++s)
          kt.push_back({t.block, t.m0, t.n0, t.kind, s * nk / ks, (s + 1) * nk / ks, slot, ks, s, npart});
        npart += ks;
      }
    }
    std::stable_sort(kt.begin(), kt.end(), [](const SplitTile &x, const SplitTile &y) {
      return (x.ke - x.kb) > (y.ke - y.kb);
    });
  }
  p->ws_bytes = off;
  p->nstiles = (int64_t)tiles.size();
  p->nkstiles = (int64_t)kt.size();
  p->nsjobs = (int)jobs.size();
  p->nsrows = ngroups;
  cudaError_t e = cudaSuccess;
  if (!tiles.empty()) {
    e = cudaMalloc((void **)&p->stiles, tiles.size() * sizeof(GTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->stiles, tiles.data(), tiles.size() * sizeof(GTile), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !kt.empty()) {
    e = cudaMalloc(&p->kstiles, kt.size() * sizeof(SplitTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->kstiles, kt.data(), kt.size() * sizeof(SplitTile), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && nslots > 0) {
    const size_t pb = (size_t)npart * 64 * 128 * sizeof(double);
    e = cudaMalloc((void **)&p->part, pb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->pcnt, nslots * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->pcnt, 0, nslots * sizeof(int));
  }
  if (e == cudaSuccess && !jobs.empty()) {
    e = cudaMalloc(&p->sjobs, jobs.size() * sizeof(SliceJob));
    if (e == cudaSuccess) e = cudaMemcpy(p->sjobs, jobs.data(), jobs.size() * sizeof(SliceJob), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->srow_begin, grp_begin.size() * 8);
    if (e == cudaSuccess) e = cudaMemcpy(p->srow_begin, grp_begin.data(), grp_begin.size() * 8, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess)
    return tkb_set_error(ctx, TKB_ERR_CUDA, std::string("split plan upload: ") + cudaGetErrorString(e));
  return tkb_ensure_workspace(ctx, p->ws_bytes);
}

int tkb_gemm_split_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A,
                          const void *B, tkb_scalar alpha, tkb_scalar beta) {
  if (p->nstiles == 0) return TKB_OK;
  if (p->dtype == TKB_F64 && (alpha.im != 0.0 || beta.im != 0.0))
    return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
  if (ctx->ws_bytes < p->ws_bytes)
    return tkb_set_error(ctx, TKB_ERR_ARG, "context workspace smaller than the plan needs");
  CDbl a{alpha.re, alpha.im}, b{beta.re, beta.im};
  switch (p->slices) {
    case 3: return launch_split<3>(ctx, p, C, A, B, a, b);
    case 4: return launch_split<4>(ctx, p, C, A, B, a, b);
    case 5: return launch_split<5>(ctx, p, C, A, B, a, b);
    case 6: return launch_split<6>(ctx, p, C, A, B, a, b);
    default: return launch_split<7>(ctx, p, C, A, B, a, b);
  }
}
