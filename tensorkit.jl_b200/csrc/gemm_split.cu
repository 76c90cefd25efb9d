// Split-precision grouped block GEMM (Ozaki scheme I on the INT8 tensor pipe).
//
// Method (Ozaki, Ogita, Oishi & Rump 2012; Ootomo, Ozaki & Yokota 2024, "DGEMM on integer
// matrix multiplication unit"): every row i of op(A) is scaled by 2^-e_i (e_i the binary
// exponent bounding the row's largest magnitude) and cut into S int8 slices,
//     A_il·2^-e_i = Σ_{s=1..S} a^(s)_il · 2^-7s + r_il,   |a^(s)| ≤ 127,  |r| ≤ 2^-(7S+1),
// the slices being the signed base-128 digits of |A_il|·2^(7S−e_i) rounded to an integer.
// Columns of op(B) are cut the same way with exponents f_j. Then
//     C_ij ≈ 2^(e_i+f_j) Σ_{d=2..S+1} 2^-7d P_d,ij ,   P_d = Σ_{s+t=d} a^(s) b^(t),
// where every P_d is an exact INT32 tensor-core accumulation (K ranges of at most
// (2^31 − 1)/(S·127²) per product task keep it exact; longer K loops are split). Terms with
// s+t > S+1 are below the truncation error and dropped. The recombination, the α/β update
// and everything after the integer products are FP64.
//
// ComplexF64 blocks are mapped to one real product: op(A) becomes the 2m×2k real matrix with
// row pairs (2r, 2r+1) = ([Re A_r, -Im A_r], [Im A_r, Re A_r]) and op(B) the 2k×n matrix
// [Re B; Im B], so rows 2r and 2r+1 of the real result are Re and Im of C_r. The two K
// halves are each zero-padded to round_up(k, 16) positions.
//
// Slice layout in the workspace: per block, the rows of op(A) (op(B)ᵀ) are cut into panels
// of 128 (64) rows; a panel is a sequence of 32-byte K stages (one tensor-core K step), and a
// stage holds the S slices one after another, each in the canonical K-major "core matrix"
// layout of the tensor-core operand descriptors (8-row × 16-byte core matrices; 256 bytes
// between 8-row groups, 128 bytes between the two 16-byte K chunks). One stage of all S
// slices of a panel is therefore one contiguous S·4 KiB (S·2 KiB) block that a single bulk
// copy moves into shared memory (the issue rate of one producer thread, not the copy size,
// limits the ring).
//
// One persistent launch per grouped GEMM (gemm_split_fused_kernel, one CTA per SM): the CTAs
// first claim slicing tasks (up to 32 source rows over the whole K range: row maxima, exponents,
// slices; the operand is read once), then run the products items (128×64 output tiles, or K
// pieces of them) with a producer warp streaming the stages of A and B with cp.async.bulk into a
// shared-memory ring as deep as fits (5 stages at S = 7), an MMA warp issuing
// tcgen05.mma.kind::i8 (M=128, K=32, N = 64 per B slice, up to four B slices per instruction)
// into S int32 diagonal accumulators held in tensor memory (S·64 of 512 columns), and eight
// epilogue warps (two per TMEM lane quarter) reading the accumulators back with tcgen05.ld and
// recombining them in FP64 while the next item's stages load.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "tkb_internal.h"

namespace {

constexpr int PANEL_A = 128, PANEL_B = 64;   // rows per panel
constexpr int KSTAGE = 32;                   // bytes of K per stage (one tensor-core K step)
constexpr int kSmemMax = 232448;             // dynamic shared memory per CTA (227 KiB)
constexpr int kSmemTail = 2048;              // barriers and small tables after the ring
// depth of the shared-memory ring: as many stages of S slices of A and B as fit, at most 8
__host__ __device__ constexpr int ring_stages(int S) {
  return (kSmemMax - kSmemTail) / (S * (PANEL_A + PANEL_B) * KSTAGE) < 8
             ? (kSmemMax - kSmemTail) / (S * (PANEL_A + PANEL_B) * KSTAGE)
             : 8;
}
constexpr int SMAX = 7;

struct CDbl {
  double x, y;
};

// 2^e as a double for e in the normal range (exact)
__device__ __forceinline__ double pow2i(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }
// out of line: the rare exponents outside the normal range must not inflate the code of the
// short-lived kernels that scale every element
__device__ __noinline__ double ldexp_slow(double v, int e) { return ldexp(v, e); }
// v·2^e: one exact multiplication when 2^e is a normal number, else ldexp
__device__ __forceinline__ double scale2(double v, int e) {
  return (e >= -1022 && e <= 1023) ? v * pow2i(e) : ldexp_slow(v, e);
}
// exact int64 → double for |x| < 2^51: x is added to the mantissa of 1.5·2^52 (whose unit in
// the last place is 1), and 1.5·2^52 is subtracted again
__device__ __forceinline__ double i2d_small(int64_t x) {
  return __longlong_as_double(x + 0x4338000000000000ll) - 6755399441055744.0;
}

// byte offset of (slice 0, row r, K byte kb) in a block's slices (pr: rows per panel, 64 or
// 128); slice s is s·pr·KSTAGE bytes further
__host__ __device__ __forceinline__ int64_t slice_off(int64_t r, int64_t kb, int64_t kpad, int pr, int S) {
  const int lpr = pr == 128 ? 7 : 6;
  const int64_t panel = r >> lpr, rr = r & (pr - 1);
  const int64_t stg = kb >> 5, kk = kb & 31;
  return (panel * kpad + stg * KSTAGE) * (int64_t)(S * pr) + (rr >> 3) * 256 + (kk >> 4) * 128 + (rr & 7) * 16 +
         (kk & 15);
}

// Slicing: one task = nrows source rows of one operand of one block over the whole K range.
// Source rows are the rows of op(A) and the columns of op(B) (for ComplexF64 a complex source row
// of op(A) gives the real row pair 2r, 2r+1). A task is cut into pieces of LK consecutive K
// values of one source row (LK = 16 real values: one 16-byte slice store; 8 complex values: one
// 8-byte store per real row and K half), dealt to the threads round-robin:
//   rows contiguous in memory (real op(A) = A, op(B) = Bᵀ; complex likewise): consecutive
//     threads take consecutive rows of one K chunk, so every load instruction of a warp reads
//     consecutive rows (coalesced);
//   K contiguous (op(A) = Aᵀ/Aᴴ, op(B) = B): consecutive threads take consecutive K chunks of
//     one row; a thread reads its chunk as 16-byte vectors when the row is aligned.
// Phase 1 loads the pieces, reduces each piece's maximum magnitude and sum of squares and
// combines them per row in shared memory; the first kSliceKeep pieces of every thread stay in
// registers, so tasks with at most kSliceKeep pieces per thread (the planner sizes them so) read
// the operand once. Phase 2 turns the row maxima into exponents and writes the S slices of every
// piece.
struct SliceTask {  // one entry per task
  int32_t block;
  int32_t operand;  // 0 = rows of op(A), 1 = columns of op(B)
  int32_t r0;       // first source row
  int32_t nrows;    // source rows of the task (≤ kSliceMaxRows)
};

constexpr int kSlicePlanThreads = 256;  // threads the planner sizes the tasks for (at least)
constexpr int kSliceKeep = 2;           // pieces per thread held in registers between the phases
constexpr int kSliceMaxRows = 32;       // source rows per task

template <int LK>
struct Piece;  // LK int8 digits: one store per slice
template <>
struct Piece<8> {
  using T = uint2;
};
template <>
struct Piece<16> {
  using T = uint4;
};

template <bool CPLX>
struct SrcVal;
template <>
struct SrcVal<false> {
  using T = double;
};
template <>
struct SrcVal<true> {
  using T = double2;
};

__device__ __forceinline__ double zero_of(double) { return 0.0; }
__device__ __forceinline__ double2 zero_of(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double absmax(double v) { return fabs(v); }
__device__ __forceinline__ double absmax(double2 v) { return fmax(fabs(v.x), fabs(v.y)); }
__device__ __forceinline__ double sq_of(double v) { return v * v; }
__device__ __forceinline__ double sq_of(double2 v) { return fma(v.x, v.x, v.y * v.y); }

// LK consecutive K values c .. c+LK−1 of the source row at element offset `base` (K stride
// ks), zero beyond ksrc or for an invalid row
template <bool CPLX, bool ROWC, int LK>
__device__ __forceinline__ void load_piece(const typename SrcVal<CPLX>::T *__restrict__ X, int64_t base,
                                           int64_t ks, int64_t c, int64_t ksrc, bool rv,
                                           typename SrcVal<CPLX>::T (&v)[LK]) {
  using T = typename SrcVal<CPLX>::T;
  const T z = zero_of(T{});
  if (!rv) {
#pragma unroll
    for (int q = 0; q < LK; ++q) v[q] = z;
    return;
  }
  const T *p = X + base + c * ks;
  if constexpr (!ROWC && !CPLX) {
    if (c + LK <= ksrc && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
      const double2 *p2 = reinterpret_cast<const double2 *>(p);
#pragma unroll
      for (int h = 0; h < LK / 2; ++h) {
        const double2 w = __ldg(p2 + h);
        v[2 * h] = w.x;
        v[2 * h + 1] = w.y;
      }
      return;
    }
  }
#pragma unroll
  for (int q = 0; q < LK; ++q) v[q] = (c + q < ksrc) ? __ldg(p + q * ks) : z;
}

// Integer slicing. The row exponent e is the binary exponent of the row maximum m
// (m = f·2^e, f in [0.5, 1)), raised by one when round(f·2^(7S)) would reach 2^(7S), so that
// Y = round(|v|·2^(7S−e)) < 2^(7S) for every v of the row. Y is read from the mantissa of
// z = fma(|v|·sa, sb, 2^52) with sa·sb = 2^(7S−e): both factors are normal powers of two,
// |v|·sa is exact, the fused multiply-add rounds once, and a double in [2^52, 2^53) holds
// z − 2^52 = Y in its low 52 bits. The S slices are the base-128 digits of Y, most
// significant first, each carrying the sign of v, so the dropped low-order products keep
// random signs (no bias across K).
template <int S>
__device__ __forceinline__ int row_exponent(double m) {
  if (!(m > 0.0)) return 0;
  int e;
  const double f = frexp(m, &e);
  return f >= 1.0 - pow2i(-(7 * S + 1)) ? e + 1 : e;
}
struct RowScale {
  double sa, sb;  // sa·sb = 2^(7S−e); sa = 1 unless 2^(7S−e) is not a normal double
};
template <int S>
__device__ __forceinline__ RowScale row_scale(int e) {
  const int t = 7 * S - e;  // in [7S − 1025, 7S + 1073]
  const int b = t <= 1000 ? t : 1000;
  return RowScale{pow2i(t - b), pow2i(b)};
}
struct Fixed {
  uint32_t hi;  // bits 32..63 of z (Y >> 32 in the low bits)
  uint32_t lo;  // Y mod 2^32
};
__device__ __forceinline__ Fixed to_fixed(double v, const RowScale &rs) {
  const double z = fma(fabs(v) * rs.sa, rs.sb, 4503599627370496.0);  // 2^52 + Y
  return Fixed{(uint32_t)__double2hiint(z), (uint32_t)__double2loint(z)};
}
// byte masks of the negative values among 4·NW (0xff per value with its sign bit set)
template <int NW, typename F>
__device__ __forceinline__ void sign_masks(F &&val, uint32_t (&M)[NW]) {
#pragma unroll
  for (int h = 0; h < NW; ++h) {
    uint32_t s[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) s[b] = (uint32_t)(__double2hiint(val(4 * h + b)) >> 31);
    M[h] = __byte_perm(__byte_perm(s[0], s[1], 0x0040), __byte_perm(s[2], s[3], 0x0040), 0x5410);
  }
}
// digit sl (0 = most significant) of LK fixed-point values as one LK-byte piece of int8:
// the 7-bit digit of Y, negated in the bytes that M marks (bytes 0..127: the negation is
// (0x80 − b) ^ 0x80, with no carry between bytes)
template <int S, int LK>
__device__ __forceinline__ typename Piece<LK>::T slice_piece(const Fixed (&x)[LK], const uint32_t (&M)[LK / 4],
                                                             int sl) {
  const int sh = 7 * (S - 1 - sl);
  uint32_t d[LK];
  if (sh >= 32) {
#pragma unroll
    for (int q = 0; q < LK; ++q) d[q] = x[q].hi >> (sh - 32);
  } else {
#pragma unroll
    for (int q = 0; q < LK; ++q) d[q] = __funnelshift_r(x[q].lo, x[q].hi, sh);
  }
  uint32_t w[LK / 4];
#pragma unroll
  for (int h = 0; h < LK / 4; ++h) {
    const uint32_t u = __byte_perm(__byte_perm(d[4 * h], d[4 * h + 1], 0x0040),
                                   __byte_perm(d[4 * h + 2], d[4 * h + 3], 0x0040), 0x5410) & 0x7f7f7f7fu;
    const uint32_t n = (0x80808080u - u) ^ 0x80808080u;
    w[h] = (u & ~M[h]) | (n & M[h]);
  }
  if constexpr (LK == 8) return make_uint2(w[0], w[1]);
  else return make_uint4(w[0], w[1], w[2], w[3]);
}

// the S slices of one piece: source row r, K values c .. c+LK−1, row exponent e
template <int S, bool CPLX, int LK>
__device__ __forceinline__ void store_piece(const typename SrcVal<CPLX>::T (&v)[LK], int op, bool conj, int64_t r,
                                            int64_t c, int64_t kfull, int64_t kpad, int8_t *base, int e) {
  const int pr = op == 0 ? PANEL_A : PANEL_B;
  const int64_t plane = (int64_t)pr * KSTAGE;  // between the slices of one stage
  const RowScale rsc = row_scale<S>(e);
  using P = typename Piece<LK>::T;
  if constexpr (!CPLX) {
    Fixed x[LK];
    uint32_t M[LK / 4];
#pragma unroll
    for (int q = 0; q < LK; ++q) x[q] = to_fixed(v[q], rsc);
    sign_masks([&](int q) { return v[q]; }, M);
    int8_t *p = base + slice_off(r, c, kpad, pr, S);
#pragma unroll
    for (int sl = 0; sl < S; ++sl) *reinterpret_cast<P *>(p + sl * plane) = slice_piece<S, LK>(x, M, sl);
  } else {
    Fixed xr[LK], xi[LK];
    uint32_t Mr[LK / 4], Mi[LK / 4], Mn[LK / 4];
#pragma unroll
    for (int q = 0; q < LK; ++q) {
      xr[q] = to_fixed(v[q].x, rsc);
      xi[q] = to_fixed(v[q].y, rsc);
    }
    sign_masks([&](int q) { return v[q].x; }, Mr);
    sign_masks([&](int q) { return conj ? -v[q].y : v[q].y; }, Mi);
    if (op == 0) {  // rows 2r: [Re | -Im], 2r+1: [Im | Re]
#pragma unroll
      for (int h = 0; h < LK / 4; ++h) Mn[h] = ~Mi[h];
      int8_t *p0 = base + slice_off(2 * r, c, kpad, pr, S);
      int8_t *p1 = base + slice_off(2 * r, kfull + c, kpad, pr, S);
      int8_t *p2 = base + slice_off(2 * r + 1, c, kpad, pr, S);
      int8_t *p3 = base + slice_off(2 * r + 1, kfull + c, kpad, pr, S);
#pragma unroll
      for (int sl = 0; sl < S; ++sl) {
        const P ur = slice_piece<S, LK>(xr, Mr, sl);
        const int64_t o = sl * plane;
        *reinterpret_cast<P *>(p0 + o) = ur;
        *reinterpret_cast<P *>(p1 + o) = slice_piece<S, LK>(xi, Mn, sl);
        *reinterpret_cast<P *>(p2 + o) = slice_piece<S, LK>(xi, Mi, sl);
        *reinterpret_cast<P *>(p3 + o) = ur;
      }
    } else {  // column j of op(B): [Re | Im]
      int8_t *p0 = base + slice_off(r, c, kpad, pr, S);
      int8_t *p1 = base + slice_off(r, kfull + c, kpad, pr, S);
#pragma unroll
      for (int sl = 0; sl < S; ++sl) {
        const int64_t o = sl * plane;
        *reinterpret_cast<P *>(p0 + o) = slice_piece<S, LK>(xr, Mr, sl);
        *reinterpret_cast<P *>(p1 + o) = slice_piece<S, LK>(xi, Mi, sl);
      }
    }
  }
}

// Block statistics the slicing leaves for the slice-count choice (per block: the largest row
// exponent of op(A) rows and of op(B) columns, biased by kExpBias so that 0 means "no nonzero
// row", and the largest row 2-norms as double bits)
constexpr int kExpBias = 4096;

// Per-row maximum and sum of squares of the lanes of a warp (all lanes call; row −1 = no value).
// The lanes holding one row form runs of consecutive lanes (a row can recur later in the warp);
// every run is reduced to its first lane with a windowed shuffle reduction keyed by the run's
// first lane, and that lane adds the run's values with one shared-memory atomic each.
__device__ __forceinline__ void warp_row_account(int row, double m, double s2, unsigned long long *rmax, double *rsq) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int rp = __shfl_up_sync(full, row, 1);
  const bool head = lane == 0 || rp != row;
  int start = head ? lane : 0;  // first lane of this lane's run: a prefix maximum of the heads
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int o = __shfl_up_sync(full, start, d);
    if (lane >= d) start = max(start, o);
  }
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int so = __shfl_down_sync(full, start, d);
    const double mo = __shfl_down_sync(full, m, d);
    const double qo = __shfl_down_sync(full, s2, d);
    if (lane + d < 32 && so == start) {
      m = fmax(m, mo);
      s2 += qo;
    }
  }
  if (head && row >= 0 && m > 0.0) {
    atomicMax(&rmax[row], (unsigned long long)__double_as_longlong(m));
    atomicAdd(&rsq[row], s2);
  }
}

// One slicing task with the NT threads of the CTA. rmax, rsq (zeroed by the caller) and rexp
// are per-row shared-memory scratch of kSliceMaxRows entries; bst receives the block statistics.
template <int S, bool CPLX, bool ROWC, int NT>
__device__ __forceinline__ void slice_task(const GBlock &b, const SliceTask &task, const void *Xv, int8_t *ws,
                                           unsigned long long *rmax, int *rexp, double *rsq,
                                           unsigned long long *bst) {
  using T = typename SrcVal<CPLX>::T;
  constexpr int LK = CPLX ? 8 : 16;
  const int tid = threadIdx.x;
  const int op = task.operand;
  const int opx = op == 0 ? b.opA : b.opB;
  const int64_t xo = op == 0 ? b.offA : b.offB;
  // strides of source rows and K in elements
  int64_t rs, ks;
  if (op == 0) {
    rs = opx == TKB_OP_N ? 1 : b.lda;
    ks = opx == TKB_OP_N ? b.lda : 1;
  } else {
    rs = opx == TKB_OP_N ? b.ldb : 1;
    ks = opx == TKB_OP_N ? 1 : b.ldb;
  }
  const bool conj = opx == TKB_OP_C;
  const int64_t msrc = op == 0 ? b.m : b.n;
  const int64_t kfull = CPLX ? b.kpad / 2 : b.kpad;
  const int nchunk = (int)(kfull / LK);
  const int nrows = task.nrows;
  const int npieces = nrows * nchunk;
  const T *X = reinterpret_cast<const T *>(Xv);
  auto piece_of = [&](int p, int &row, int64_t &c) {
    if (ROWC) {
      row = p % nrows;
      c = (int64_t)(p / nrows) * LK;
    } else {
      row = p / nchunk;
      c = (int64_t)(p % nchunk) * LK;
    }
  };
  auto load = [&](int p, T (&v)[LK], int &row, int64_t &c) {
    piece_of(p, row, c);
    const int64_t r = task.r0 + row;
    load_piece<CPLX, ROWC, LK>(X, xo + r * rs, ks, c, b.k, r < msrc, v);
  };
  // a piece's maximum magnitude and sum of squares, combined per row: first over the runs of
  // lanes of the warp that hold the same row (every lane takes part; lanes without a piece pass
  // row −1), then one shared-memory atomic per run
  auto account = [&](const T (&v)[LK], int row, bool active) {
    double m = 0.0, s2 = 0.0;
    if (active) {
#pragma unroll
      for (int l = 0; l < LK; ++l) {
        m = fmax(m, absmax(v[l]));
        s2 += sq_of(v[l]);
      }
    } else {
      row = -1;
    }
    warp_row_account(row, m, s2, rmax, rsq);
  };

  // phase 1: row maxima and sums of squares; the first kSliceKeep pieces stay in registers
  // (the loops run warp-uniformly: every lane of a warp reaches the warp reductions together)
  const int wbase = tid & ~31, lane = tid & 31;
  T keep[kSliceKeep][LK];
#pragma unroll
  for (int q = 0; q < kSliceKeep; ++q) {
    const int p = tid + q * NT;
    int row = 0;
    int64_t c = 0;
    const bool act = p < npieces;
    if (act) load(p, keep[q], row, c);
    account(keep[q], row, act);
  }
  for (int p0 = wbase + kSliceKeep * NT; p0 < npieces; p0 += NT) {
    const int p = p0 + lane;
    T v[LK];
    int row = 0;
    int64_t c = 0;
    const bool act = p < npieces;
    if (act) load(p, v, row, c);
    account(v, row, act);
  }
  __syncthreads();
  if (tid < 32) {  // nrows ≤ 32: one warp finishes the rows
    const int64_t r = task.r0 + tid;
    const double m = tid < nrows ? __longlong_as_double((long long)rmax[tid]) : 0.0;
    const int e = row_exponent<S>(m);
    if (tid < nrows) rexp[tid] = e;
    if (tid < nrows && r < msrc) {
      int32_t *ex = reinterpret_cast<int32_t *>(ws + (op == 0 ? b.wsEA : b.wsEB));
      if (CPLX && op == 0) {
        ex[2 * r] = e;
        ex[2 * r + 1] = e;
      } else {
        ex[r] = e;
      }
    }
    // block statistics: largest exponent and 2-norm among the task's nonzero rows
    const unsigned eb = (m > 0.0) ? (unsigned)(e + kExpBias) : 0u;
    double nrm = (m > 0.0) ? sqrt(rsq[tid]) : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nrm = fmax(nrm, __shfl_xor_sync(0xffffffffu, nrm, o));
    const unsigned ebm = __reduce_max_sync(0xffffffffu, eb);
    if (tid == 0 && ebm != 0u) {
      atomicMax(&bst[4 * task.block + op], (unsigned long long)ebm);
      atomicMax(&bst[4 * task.block + 2 + op], (unsigned long long)__double_as_longlong(nrm));
    }
  }
  __syncthreads();

  // phase 2: slices (rows beyond the operand are not written: their outputs are discarded)
  int8_t *base = ws + (op == 0 ? b.wsA : b.wsB);
#pragma unroll
  for (int q = 0; q < kSliceKeep; ++q) {
    const int p = tid + q * NT;
    if (p < npieces) {
      int row;
      int64_t c;
      piece_of(p, row, c);
      const int64_t r = task.r0 + row;
      if (r < msrc) store_piece<S, CPLX, LK>(keep[q], op, conj, r, c, kfull, b.kpad, base, rexp[row]);
    }
  }
  for (int p = tid + kSliceKeep * NT; p < npieces; p += NT) {
    T v[LK];
    int row;
    int64_t c;
    load(p, v, row, c);
    const int64_t r = task.r0 + row;
    if (r < msrc) store_piece<S, CPLX, LK>(v, op, conj, r, c, kfull, b.kpad, base, rexp[row]);
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
// tcgen05.ld of 8 columns without the wait; tmem_ld_wait8 on the same registers orders their
// uses after it
__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait8(uint32_t (&r)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
               :
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

constexpr uint32_t kTmemCols = 512;
// instruction descriptor: D s32 (bits 4-5 = 2), A/B signed int8 (bits 7-9, 10-12 = 1),
// both K-major, N (bits 17-22 = N>>3), M = 128 (bits 24-28 = 128>>4)
__host__ __device__ constexpr uint32_t idesc_i8(uint32_t n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}
// B slices per product: the products (s, t), (s, t+1), … share the A slice s and land in the
// adjacent diagonals s+t, s+t+1, … of TMEM; the B slices of a stage lie back to back (2 KiB,
// i.e. 64 rows, each, with the same 256-byte step between 8-row groups), so up to four of them
// form one N ≤ 256 operand and one instruction computes the four products.
constexpr int kMaxSlicesPerMma = 4;


// One products item: output tile (m0, n0) of a block, K stages [kb, ke); kind 0 = products,
// 1 = β-scale only (k = 0). When a tile's K range is split into nsplit pieces (few tiles, long
// K), each piece recombines its own int32 diagonals into an FP64 partial tile in partial buffer
// pbase + sid, and the piece that arrives last on counter `slot` adds the partials in piece
// order (deterministic) before the check, the α/β update and the store to C.
struct SplitTile {
  int32_t block, m0, n0, kind;
  int32_t kb, ke, slot, nsplit;
  int32_t sid, pbase;
};

// ---- slice count per block and the FP64 check -----------------------------------------------
// The S-slice product of one output C_ij = Σ_k a_ik b_kj has an error that behaves like a sum of
// K terms of random sign (rounded digits, dropped low products) of size about
// 2^(e_i + f_j − 7S), so its spread grows like √(S·K)·2^(e_i + f_j − 7S). The slicing records,
// per block, the largest row exponent of op(A) and of op(B) (e, f) and the largest row 2-norms
// (‖a‖, ‖b‖); the typical largest |C_ij| of a block is then about 4.5·‖a‖·‖b‖/√K. A block gets the
// smallest S in [3, S_max] with
//     kGuardSigma · √(S·K) · 2^(e + f − 7S)  ≤  kSliceTol · kSliceMargin · 4.5·‖a‖·‖b‖/√K,
// (S_max = 7 by default; a caller that fixes the slice count gets exactly that count for every
// block and no check)
// the expected largest error within the tolerance with margin to spare. Rows and columns whose
// exponent range is wide (one entry far above the rest, so ‖a‖ is close to max|a| and the other
// entries keep few significant bits) push S up; a block that no S ≤ S_max serves is computed in
// FP64. Smaller S use the leading digits of the S_max-digit slices.
// Cancellation (C far smaller than |A|·|B|) is invisible to these statistics, so every tile is
// checked after its products: with its own largest exponents and largest |C|, a tile whose
// estimate kGuardSigma·√(S·K)·2^(e + f − 7S) exceeds kSliceTol·max|C_tile| is recomputed in FP64
// (DMMA) by the epilogue warps. These are statistical estimates, not rigorous bounds; the tests
// check the errors they admit against the FP64 oracle.
constexpr double kSliceTol = 1e-12;
constexpr double kGuardSigma = 1.5;
constexpr double kSliceMargin = 0.5;

template <int SM>
__device__ __forceinline__ int choose_slices(const unsigned long long *bst, int block, int64_t kpad) {
  const unsigned long long ea = bst[4 * block], eb = bst[4 * block + 1];
  if (ea == 0ull || eb == 0ull) return SM;  // an operand of the block is zero: so are its products
  const double na = __longlong_as_double((long long)bst[4 * block + 2]);
  const double nb = __longlong_as_double((long long)bst[4 * block + 3]);
  const double k = (double)kpad;
  const double cmax = 4.5 * na * nb / sqrt(k);
  const int e = (int)ea + (int)eb - 2 * kExpBias;
  for (int s = 3; s <= SM; ++s) {
    const double est = kGuardSigma * sqrt((double)s * k) * ldexp(1.0, e - 7 * s);
    if (est <= kSliceTol * kSliceMargin * cmax) return s;
  }
  return 0;
}

// FP64 DMMA (the fallback of tiles and blocks that the slices do not serve)
__device__ __forceinline__ void dmma_f64(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// one element of op(A) / op(B) of a block straight from the FP64 operands (zero outside)
template <bool CPLX>
__device__ __forceinline__ typename SrcVal<CPLX>::T opA_at(const GBlock &b, const void *A, int64_t i, int64_t l) {
  using T = typename SrcVal<CPLX>::T;
  if (i >= b.m || l >= b.k) return zero_of(T{});
  const T *X = reinterpret_cast<const T *>(A) + b.offA;
  T v = b.opA == TKB_OP_N ? X[i + l * b.lda] : X[l + i * b.lda];
  if constexpr (CPLX) {
    if (b.opA == TKB_OP_C) v.y = -v.y;
  }
  return v;
}
template <bool CPLX>
__device__ __forceinline__ typename SrcVal<CPLX>::T opB_at(const GBlock &b, const void *B, int64_t l, int64_t j) {
  using T = typename SrcVal<CPLX>::T;
  if (j >= b.n || l >= b.k) return zero_of(T{});
  const T *X = reinterpret_cast<const T *>(B) + b.offB;
  T v = b.opB == TKB_OP_N ? X[l + j * b.ldb] : X[j + l * b.ldb];
  if constexpr (CPLX) {
    if (b.opB == TKB_OP_C) v.y = -v.y;
  }
  return v;
}

// FP64 fallback: the eight epilogue warps compute one whole output tile with DMMA
// (mma.sync.m8n8k4.f64) from the FP64 operands over the full K range, and store α·C + β·C_old.
// Real: tile rows m0 .. m0+127, warp (w mod 4, w / 4) takes 32 rows × 32 columns. Complex: the
// tile's real row pairs are complex rows m0/2 .. m0/2+63; a warp takes 16 complex rows × 32
// columns, four real DMMA per complex product.
template <bool CPLX>
__device__ __noinline__ void fp64_tile(const GBlock &b, int64_t m0, int64_t n0, const void *A, const void *B,
                                       double *C, CDbl alpha, CDbl beta, bool bz, int warp, int lane) {
  const int g8 = lane >> 2, t4 = lane & 3;
  if constexpr (!CPLX) {
    const int64_t r0 = m0 + 32 * (warp & 3), c0 = n0 + 32 * (warp >> 2);
    double acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.0;
    for (int64_t k0 = 0; k0 < b.k; k0 += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = opA_at<false>(b, A, r0 + 8 * mi + g8, k0 + t4);
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = opB_at<false>(b, B, k0 + t4, c0 + 8 * ni + g8);
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma_f64(acc[(mi * 4 + ni) * 2], acc[(mi * 4 + ni) * 2 + 1], af[mi], bf[ni]);
    }
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      const int mi = q / 8, ni = (q / 2) % 4, h = q % 2;
      const int64_t i = r0 + 8 * mi + g8, j = c0 + 8 * ni + 2 * t4 + h;
      if (i < b.m && j < b.n) {
        double *p = C + b.offC + i + j * b.ldc;
        const double r = alpha.x * acc[q];
        *p = bz ? r : fma(beta.x, *p, r);
      }
    }
  } else {
    const int64_t r0 = m0 / 2 + 16 * (warp & 3), c0 = n0 + 32 * (warp >> 2);
    double acc[32];  // [(mi·4 + ni)·4 + {0,1}] real parts of columns 2t, 2t+1; + {2,3} imaginary
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.0;
    for (int64_t k0 = 0; k0 < b.k; k0 += 4) {
      double2 af[2], bf[4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) af[mi] = opA_at<true>(b, A, r0 + 8 * mi + g8, k0 + t4);
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = opB_at<true>(b, B, k0 + t4, c0 + 8 * ni + g8);
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          double *a = &acc[(mi * 4 + ni) * 4];
          dmma_f64(a[0], a[1], af[mi].x, bf[ni].x);
          dmma_f64(a[0], a[1], -af[mi].y, bf[ni].y);
          dmma_f64(a[2], a[3], af[mi].x, bf[ni].y);
          dmma_f64(a[2], a[3], af[mi].y, bf[ni].x);
        }
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t i = r0 + 8 * mi + g8, j = c0 + 8 * ni + 2 * t4 + h;
          if (i < b.m && j < b.n) {
            double2 *p = reinterpret_cast<double2 *>(C) + b.offC + i + j * b.ldc;
            const double vr = acc[(mi * 4 + ni) * 4 + h], vi = acc[(mi * 4 + ni) * 4 + 2 + h];
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

// ---- fused persistent kernel: slicing + products + recombination in one launch ------------
// One CTA per SM (the ring fills shared memory, the accumulators most of TMEM):
//   phase 1: the CTAs claim slicing tasks from a device counter (so every task is taken by a
//     running CTA) and slice them with all warps; each finished task adds its rows to the
//     readiness count of its (block, operand) after recording the block statistics;
//   phase 2: CTA b takes the products items b, b + G, ... (tiles and split-K pieces in decreasing
//     length). Once a block's operands are sliced (readiness counts, bounded waits) every role
//     derives the block's slice count S_b from the statistics, then:
//       warp 8 (one lane) streams the leading S_b slices of each K stage into the ring with
//         cp.async.bulk;
//       warp 9 (one lane) waits until the epilogue has read the previous item's accumulators,
//         issues the tcgen05 MMAs of the S_b(S_b+1)/2 products of every stage and commits;
//       warps 0-7, the epilogue (two warps per TMEM lane quarter, 32 columns each), read both
//         16-column chunks of the S_b diagonals, hand TMEM back to the MMA warp, recombine in
//         FP64, check the tile against the error estimate and store (or recompute the tile in
//         FP64 when the check fails, or when the block has S_b = 0).
//   A piece of a split tile stores its FP64 partial; the piece that arrives last on the tile's
//   counter adds the partials in piece order (deterministic), checks and stores. No CTA waits
//   for another CTA except through the readiness counts, whose slicing tasks were all claimed by
//   running CTAs, so the kernel needs no co-residency guarantee.
// The last CTA to finish records the slice counts of the launch and the number of tiles the
// check sent to FP64, and clears the claim, readiness, statistics and finish counters.
constexpr int kFusedThreads = 320;
constexpr int kEpiWarps = 8;
constexpr int kProducerWarp = 8, kMmaWarp = 9;
constexpr int kEpiBarrier = 1;  // named barrier of the 256 epilogue threads

struct FusedArgs {
  const GBlock *blocks;
  const SliceTask *stasks;
  const SplitTile *items;
  const double *A, *B;
  double *C;
  int8_t *ws;
  int *cnt;                 // [0] slicing claims, [1] finished CTAs, [2] tiles recomputed in FP64,
                            // [3 + 2·block + operand] rows sliced, [3 + 2·nblocks + slot] split-K arrivals
  unsigned long long *bst;  // 4 per block: statistics of the slicing
  int *slices_out;          // per block: the slice count of the last launch (0 = FP64, −1 = no
                            // products), then the number of tiles the check sent to FP64
  double *part;             // split-K partial tiles, [col][row] per piece
  int *err;
  CDbl alpha, beta;
  int nstasks, nitems, nblocks;
  int fixed;                // 1: the caller fixed the slice count (every block uses S, no check)
};

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// bounded wait until *p ≥ target (acquire at GPU scope); false once 2 s have passed or the CTA
// aborts
__device__ __forceinline__ bool wait_at_least(const int *p, int target, const volatile int *abort) {
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    if (ld_acquire(p) >= target) return true;
    if (*abort || globaltimer_ns() - t0 > 2000000000ull) return false;
    __nanosleep(64);
  }
}
// bounded mbarrier wait that also gives up when the CTA aborts
__device__ __forceinline__ bool mbar_wait_abortable(uint64_t *bar, uint32_t parity, const volatile int *abort) {
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
    if (*abort || globaltimer_ns() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void epi_sync() {
  asm volatile("bar.sync %0, %1;\n" ::"n"(kEpiBarrier), "n"(kEpiWarps * 32) : "memory");
}
// true on every epilogue thread when it is true on any (a named-barrier reduction: the epilogue
// warps take every branch that contains a named barrier together)
__device__ __forceinline__ bool epi_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(kEpiBarrier), "n"(kEpiWarps * 32)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;\n" ::: "memory");
}

// the exact FP64 value of the first Sb int32 diagonals of one output (Horner in base 128 over
// three int64 groups, each below 2^46, then scaled and summed in FP64)
template <int S, int W>
__device__ __forceinline__ double recombine_value(const uint32_t (&r)[S][W], int q, int Sb) {
  int64_t g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
  for (int d = 0; d < S; ++d) {
    if (d < Sb) {
      const int64_t pd = (int32_t)r[d][q];
      if (d < 3) g0 = g0 * 128 + pd;
      else if (d < 5) g1 = g1 * 128 + pd;
      else g2 = g2 * 128 + pd;
    }
  }
  double acc = i2d_small(g0) * pow2i(-7 * ((Sb < 3 ? Sb : 3) + 1));
  if (Sb > 3) acc = fma(i2d_small(g1), pow2i(-7 * ((Sb < 5 ? Sb : 5) + 1)), acc);
  if (Sb > 5) acc = fma(i2d_small(g2), pow2i(-7 * (Sb + 1)), acc);
  return acc;
}

// the α/β update and store of 16 values of one row (one column chunk); real or complex rows
template <bool CPLX>
__device__ __forceinline__ void store_chunk(const double (&v)[16], int64_t i, int64_t j0, const GBlock &b, double *C,
                                            CDbl alpha, CDbl beta, bool bz) {
  if constexpr (!CPLX) {
    const int nj = (int)min((int64_t)16, b.n - j0);
    if (i >= b.m || nj <= 0) return;
    double *pc = C + b.offC + i + j0 * b.ldc;
    double old[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) old[q] = (!bz && q < nj) ? pc[q * b.ldc] : 0.0;
#pragma unroll
    for (int q = 0; q < 16; ++q)
      if (q < nj) pc[q * b.ldc] = bz ? alpha.x * v[q] : fma(beta.x, old[q], alpha.x * v[q]);
  } else {
#pragma unroll
    for (int q = 0; q < 16; ++q) store_out(v[q], i, j0 + q, b, 1, C, alpha, beta, bz, 1);
  }
}

template <int S, bool CPLX, bool BZ>
__global__ void __launch_bounds__(kFusedThreads, 1) gemm_split_fused_kernel(const FusedArgs args) {
  constexpr uint32_t A_BYTES = S * PANEL_A * KSTAGE, B_BYTES = S * PANEL_B * KSTAGE;
  constexpr uint32_t A_SLICE = PANEL_A * KSTAGE, B_SLICE = PANEL_B * KSTAGE;
  constexpr uint32_t STAGE = A_BYTES + B_BYTES;
  constexpr int NSTAGE = ring_stages(S);
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * STAGE);
  uint64_t *empty = full + NSTAGE;
  uint64_t *acc_full = full + 2 * NSTAGE;
  uint64_t *acc_empty = acc_full + 1;
  uint64_t *drain = acc_full + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_full + 3);
  int *claim = reinterpret_cast<int *>(acc_full + 4);  // [0..1] slicing claims (double-buffered), [2] ticket
  volatile int *abort = claim + 3;
  unsigned long long *rmax = reinterpret_cast<unsigned long long *>(acc_full + 6);  // kSliceMaxRows
  double *rsq = reinterpret_cast<double *>(rmax + kSliceMaxRows);                   // kSliceMaxRows
  int *rexp = reinterpret_cast<int *>(rsq + kSliceMaxRows);                         // kSliceMaxRows
  // tile check: per epilogue warp, largest |C|, row exponent and column exponent (two buffers)
  double *gmax = reinterpret_cast<double *>(rexp + kSliceMaxRows);  // [2][kEpiWarps]
  int *gexp = reinterpret_cast<int *>(gmax + 2 * kEpiWarps);        // [2][kEpiWarps][2]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const FusedArgs &g = args;
  int *ready = g.cnt + 3;
  int *arrive = g.cnt + 3 + 2 * g.nblocks;

  if (tid == 0) {
#pragma unroll
    for (int st = 0; st < NSTAGE; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kEpiWarps);
    mbar_init(drain, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  pdl_wait();  // operands and C come from earlier kernels of the stream

  // ---- phase 1: slicing tasks, claimed from the device counter ----------------------------
  if (tid == 0) claim[0] = atomicAdd(&g.cnt[0], 1);
  __syncthreads();
  int t = claim[0];
  for (int it = 0; t < g.nstasks; ++it) {
    const int nb = (it + 1) & 1;
    if (tid == 0) claim[nb] = atomicAdd(&g.cnt[0], 1);  // the next claim is in flight meanwhile
    if (tid < kSliceMaxRows) {
      rmax[tid] = 0ull;
      rsq[tid] = 0.0;
    }
    const SliceTask task = g.stasks[t];
    const GBlock &b = g.blocks[task.block];
    __syncthreads();
    const int op = task.operand;
    const int opx = op == 0 ? b.opA : b.opB;
    const bool rowc = op == 0 ? opx == TKB_OP_N : opx != TKB_OP_N;
    const void *X = op == 0 ? (const void *)g.A : (const void *)g.B;
    if (rowc) slice_task<S, CPLX, true, kFusedThreads>(b, task, X, g.ws, rmax, rexp, rsq, g.bst);
    else slice_task<S, CPLX, false, kFusedThreads>(b, task, X, g.ws, rmax, rexp, rsq, g.bst);
    // the slices are read by bulk copies (async proxy) of other CTAs: fence, then publish
    fence_proxy_async_global();
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(&ready[2 * task.block + op], task.nrows);
    }
    t = claim[nb];
  }

  // ---- phase 2: products ------------------------------------------------------------------
  const int G = gridDim.x;
  // wait (bounded) until both operands of the item's block are sliced; then its slice count
  auto block_slices = [&](const GBlock &b, int block, int &sb) -> bool {
    if (!wait_at_least(&ready[2 * block], (int)b.m, abort) || !wait_at_least(&ready[2 * block + 1], (int)b.n, abort))
      return false;
    sb = g.fixed ? S : choose_slices<S>(g.bst, block, b.kpad);
    return true;
  };
  if (warp == kProducerWarp) {
    if (lane == 0) {
      int issued = 0, landed = 0;  // stages issued / known to have landed (for the final drain)
      int gs = 0;                  // ring stage counter over all items of this CTA
      for (int ii = blockIdx.x; ii < g.nitems && !*abort; ii += G) {
        const SplitTile it = g.items[ii];
        if (it.kind != 0) continue;
        const GBlock b = g.blocks[it.block];
        int sb = 0;
        if (!block_slices(b, it.block, sb)) {
          atomicExch(g.err, 3);
          *abort = 1;
          break;
        }
        if (sb == 0) continue;  // the block runs in FP64
        fence_proxy_async_global();
        const int8_t *gA = g.ws + b.wsA + (int64_t)(it.m0 / PANEL_A) * S * PANEL_A * b.kpad;
        const int8_t *gB = g.ws + b.wsB + (int64_t)(it.n0 / PANEL_B) * S * PANEL_B * b.kpad;
        bool ok = true;
        for (int kt = it.kb; kt < it.ke; ++kt, ++gs) {
          const int st = gs % NSTAGE, n = gs / NSTAGE;
          if (n > 0) {
            if (!mbar_wait_abortable(&empty[st], (n - 1) & 1, abort)) {
              atomicExch(g.err, 1);
              *abort = 1;
              ok = false;
              break;
            }
            ++landed;  // the products of stage gs − NSTAGE are done, so it had landed
          }
          // the leading sb slices of the stage (a stage keeps its slices one after another)
          unsigned char *sa = smem + st * STAGE;
          mbar_expect_tx(&full[st], (uint32_t)sb * (A_SLICE + B_SLICE));
          bulk_g2s(sa, gA + (int64_t)kt * A_BYTES, (uint32_t)sb * A_SLICE, &full[st]);
          bulk_g2s(sa + A_BYTES, gB + (int64_t)kt * B_BYTES, (uint32_t)sb * B_SLICE, &full[st]);
          ++issued;
        }
        if (!ok) break;
      }
      // every bulk copy must land before the CTA can exit (bounded)
      for (int k = landed; k < issued; ++k) mbar_wait(&full[k % NSTAGE], (k / NSTAGE) & 1);
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      int gs = 0, li = 0;
      bool ok = true;
      for (int ii = blockIdx.x; ii < g.nitems && ok && !*abort; ii += G) {
        const SplitTile it = g.items[ii];
        if (it.kind != 0) continue;
        const GBlock b = g.blocks[it.block];
        int sb = 0;
        if (!block_slices(b, it.block, sb)) {
          atomicExch(g.err, 3);
          *abort = 1;
          break;
        }
        if (sb == 0) continue;
        if (li > 0 && !mbar_wait_abortable(acc_empty, (li - 1) & 1, abort)) {
          atomicExch(g.err, 2);
          *abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t ring0 = smem_u32(smem);
        for (int kt = it.kb; kt < it.ke; ++kt, ++gs) {
          const int st = gs % NSTAGE;
          if (!mbar_wait_abortable(&full[st], (gs / NSTAGE) & 1, abort)) {
            atomicExch(g.err, 1);
            *abort = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = ring0 + st * STAGE, b0 = a0 + A_BYTES;
          // the products (s, t), (s, t+1), … share the A slice s and land in the adjacent
          // diagonals s+t, …; up to four B slices (back to back in the stage) form one N ≤ 256
          // operand
#pragma unroll
          for (int s = 0; s < S; ++s) {
            if (s < sb) {
              const uint64_t ad = umma_desc(a0 + s * A_SLICE, 128, 256);
#pragma unroll
              for (int tt = 0; tt < S - s; tt += kMaxSlicesPerMma) {
                if (tt < sb - s) {
                  const int nsl = (sb - s - tt) < kMaxSlicesPerMma ? (sb - s - tt) : kMaxSlicesPerMma;
                  umma_i8(tmem + (uint32_t)((s + tt) * 64), ad, umma_desc(b0 + tt * B_SLICE, 128, 256),
                          idesc_i8(64u * (uint32_t)nsl), (kt > it.kb || s > 0) ? 1u : 0u);
                }
              }
            }
          }
          umma_commit(&empty[st]);
        }
        if (!ok) break;
        umma_commit(acc_full);
        ++li;
      }
      // every MMA issued by this thread completes before TMEM is released (bounded)
      umma_commit(drain);
      mbar_wait(drain, 0);
    }
    __syncwarp();
  } else {
    // epilogue warps: warp w owns TMEM lanes 32(w mod 4) .. +31 (its rows) and the column chunks
    // 2·half, 2·half + 1 of 16 columns, half = w / 4
    const int quarter = warp & 3, half = warp >> 2;
    const int row = 32 * quarter + lane;
    constexpr bool bz = BZ;
    int li = 0, gi = 0;
    for (int ii = blockIdx.x; ii < g.nitems; ii += G) {
      const SplitTile it = g.items[ii];
      const GBlock b = g.blocks[it.block];
      const int64_t Mreal = CPLX ? 2 * b.m : b.m;
      const int64_t i = it.m0 + row;
      const bool prod = it.kind == 0;
      bool stop = *abort != 0;
      int sb = 0;
      if (prod && !stop) {
        // lane 0 acquires the readiness counts; __syncwarp orders the other lanes' reads of the
        // statistics and exponents after that acquire
        if (lane == 0) stop = !block_slices(b, it.block, sb);
        __syncwarp();
        stop = __shfl_sync(0xffffffffu, stop ? 1 : 0, 0) != 0;
        sb = g.fixed ? S : choose_slices<S>(g.bst, it.block, b.kpad);
      }
      const bool mma = prod && sb > 0;  // the tile's products ran on the tensor cores
      if (mma && !stop) stop = !mbar_wait_abortable(acc_full, li & 1, abort);
      if (epi_any(stop)) {  // every epilogue warp leaves the loop here, together
        if (tid == 0) {
          atomicExch(g.err, 2);
          *abort = 1;
        }
        break;
      }
      if (prod && !mma) {
        // FP64 block: one piece (the first) computes the whole tile over the full K range
        if (it.sid == 0) fp64_tile<CPLX>(b, it.m0, it.n0, g.A, g.B, g.C, g.alpha, g.beta, bz, warp, lane);
        continue;
      }
      const bool split = it.nsplit > 1;
      double v[2][16];
#pragma unroll
      for (int cc = 0; cc < 2; ++cc)
#pragma unroll
        for (int q = 0; q < 16; ++q) v[cc][q] = 0.0;
      double vmax = 0.0;    // largest |C| of the thread's values (stored already: β = 0, unsplit)
      int ei = 0, ejm = 0;  // the thread's row exponent, the largest column exponent of its chunks
      if (mma) {
        tc_fence_after();
        const int32_t *eA = reinterpret_cast<const int32_t *>(g.ws + b.wsEA);
        const int32_t *eB = reinterpret_cast<const int32_t *>(g.ws + b.wsEB);
        ei = i < Mreal ? max(eA[i], -1100) : -1100;
        const double rscale = (ei >= -1022 && ei <= 1023) ? pow2i(ei) : 0.0;
        ejm = -1100;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int c = 2 * half + cc;
          // this lane's column of the chunk: exponent and scale, shared with the warp by shuffles
          const int64_t jl = it.n0 + c * 16 + (lane & 15);
          const int ej = jl < b.n ? max(eB[jl], -1100) : -1100;
          ejm = max(ejm, ej);
          const double cs = (ej >= -1022 && ej <= 1023) ? pow2i(ej) : 0.0;
          // the chunk in two halves of 8 columns (fewer live registers); after the last load of
          // the second chunk the accumulators go back to the MMA warp
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            uint32_t r[S][8];
#pragma unroll
            for (int d = 0; d < S; ++d)
              if (d < sb)
                tmem_ld8_issue(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(d * 64 + c * 16 + hh * 8), r[d]);
#pragma unroll
            for (int d = 0; d < S; ++d)
              if (d < sb) tmem_ld_wait8(r[d]);
            if (cc == 1 && hh == 1) {
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(acc_empty);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) v[cc][hh * 8 + q] = recombine_value<S, 8>(r, q, sb);
          }
          const bool slow = __any_sync(0xffffffffu, rscale == 0.0 || cs == 0.0);
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int ejq = __shfl_sync(0xffffffffu, ej, q);
            const double csq = __shfl_sync(0xffffffffu, cs, q);
            v[cc][q] = slow ? scale2(v[cc][q], ei + ejq) : v[cc][q] * rscale * csq;
          }
          if (BZ && !split) {
            // β = 0: store at once (no old value of C is needed should the tile check send the
            // tile to FP64, which then overwrites it), keep only the largest magnitude
#pragma unroll
            for (int q = 0; q < 16; ++q) vmax = fmax(vmax, fabs(v[cc][q]));
            store_chunk<CPLX>(v[cc], i, it.n0 + c * 16, b, g.C, g.alpha, g.beta, true);
          }
        }
        ++li;
      }
      bool final_piece = true;
      if (split) {
        // store this piece's partial and count it; the last piece adds all partials in piece order
        double *mine = g.part + (int64_t)(it.pbase + it.sid) * (64 * 128);
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
#pragma unroll
          for (int q = 0; q < 16; ++q) __stcg(&mine[((2 * half + cc) * 16 + q) * 128 + row], v[cc][q]);
        __threadfence();
        epi_sync();
        if (tid == 0) claim[2] = atomicAdd(&arrive[it.slot], 1);
        epi_sync();
        final_piece = claim[2] == it.nsplit - 1;
        epi_sync();  // the ticket slot is rewritten by the next item
        if (final_piece) {
          __threadfence();
#pragma unroll
          for (int cc = 0; cc < 2; ++cc)
#pragma unroll
            for (int q = 0; q < 16; ++q) v[cc][q] = 0.0;
#pragma unroll 1
          for (int sp = 0; sp < it.nsplit; ++sp) {
            const double *src = g.part + (int64_t)(it.pbase + sp) * (64 * 128);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
              for (int q = 0; q < 16; ++q) v[cc][q] += __ldcg(&src[((2 * half + cc) * 16 + q) * 128 + row]);
          }
          if (tid == 0) arrive[it.slot] = 0;  // every piece has arrived: free for the next launch
        }
      }
      if (!final_piece) continue;  // uniform: every epilogue thread read the same ticket
      if (!mma) {                  // β-scale only (k = 0)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
          store_chunk<CPLX>(v[cc], i, it.n0 + (2 * half + cc) * 16, b, g.C, g.alpha, g.beta, bz);
        continue;
      }
      // tile check: largest |C| and exponents of the tile against the error estimate
      const bool stored = BZ && !split;
      double vm = vmax;
      if (!stored) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
#pragma unroll
          for (int q = 0; q < 16; ++q) vm = fmax(vm, fabs(v[cc][q]));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
      const int eim = (int)__reduce_max_sync(0xffffffffu, (unsigned)(ei + kExpBias)) - kExpBias;
      const int ejw = (int)__reduce_max_sync(0xffffffffu, (unsigned)(ejm + kExpBias)) - kExpBias;
      const int buf = gi & 1;
      if (lane == 0) {
        gmax[buf * kEpiWarps + warp] = vm;
        gexp[(buf * kEpiWarps + warp) * 2] = eim;
        gexp[(buf * kEpiWarps + warp) * 2 + 1] = ejw;
      }
      epi_sync();
      double tmax = 0.0;
      int te = -1100, tf = -1100;
#pragma unroll
      for (int w = 0; w < kEpiWarps; ++w) {
        tmax = fmax(tmax, gmax[buf * kEpiWarps + w]);
        te = max(te, gexp[(buf * kEpiWarps + w) * 2]);
        tf = max(tf, gexp[(buf * kEpiWarps + w) * 2 + 1]);
      }
      ++gi;
      const double est = kGuardSigma * sqrt((double)sb * (double)b.kpad) * ldexp(1.0, te + tf - 7 * sb);
      if (!g.fixed && est > kSliceTol * tmax) {  // uniform over the epilogue warps
        if (tid == 0) atomicAdd(&g.cnt[2], 1);
        if (stored) epi_sync();  // every approximate value of the tile is stored before the overwrite
        fp64_tile<CPLX>(b, it.m0, it.n0, g.A, g.B, g.C, g.alpha, g.beta, bz, warp, lane);
        continue;
      }
      if (!stored) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
          store_chunk<CPLX>(v[cc], i, it.n0 + (2 * half + cc) * 16, b, g.C, g.alpha, g.beta, bz);
      }
    }
  }

  // ---- teardown ----------------------------------------------------------------------------
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
  }
  if (tid == 0) {
    // the last CTA out records the launch's slice counts and checks, and clears the counters
    __threadfence();
    if (atomicAdd(&g.cnt[1], 1) == (int)gridDim.x - 1) {
      __threadfence();
      for (int q = 0; q < g.nblocks; ++q) {
        const GBlock &b = g.blocks[q];
        g.slices_out[q] = (b.m > 0 && b.n > 0 && b.k > 0 && !b.skinny) ? (g.fixed ? S : choose_slices<S>(g.bst, q, b.kpad))
                                                                        : -1;
      }
      g.slices_out[g.nblocks] = g.cnt[2];
      g.cnt[0] = 0;
      g.cnt[2] = 0;
      for (int q = 0; q < 2 * g.nblocks; ++q) ready[q] = 0;
      for (int q = 0; q < 4 * g.nblocks; ++q) g.bst[q] = 0ull;
      __threadfence();
      g.cnt[1] = 0;
    }
  }
}

size_t tc_smem_bytes(int S) { return ring_stages(S) * (size_t)S * (PANEL_A + PANEL_B) * KSTAGE + kSmemTail; }

template <int S>
int launch_split(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B, CDbl a, CDbl b) {
  const bool cplx = p->dtype == TKB_C128;
  FusedArgs fa;
  fa.blocks = p->blocks;
  fa.stasks = (const SliceTask *)p->sjobs;
  fa.items = (const SplitTile *)p->kstiles;
  fa.A = (const double *)A;
  fa.B = (const double *)B;
  fa.C = (double *)C;
  fa.ws = (int8_t *)ctx->ws;
  fa.cnt = p->pcnt;
  fa.bst = p->bstat;
  fa.slices_out = p->bslices;
  fa.part = p->part;
  fa.err = ctx->counters + 8;
  fa.alpha = a;
  fa.beta = b;
  fa.nstasks = (int)p->nsrows;
  fa.nitems = (int)p->nkstiles;
  fa.nblocks = (int)p->hblocks.size();
  fa.fixed = p->slices_fixed;
  const size_t smem = tc_smem_bytes(S);
  const bool bz = b.x == 0.0 && b.y == 0.0;
  auto k = cplx ? (bz ? gemm_split_fused_kernel<S, true, true> : gemm_split_fused_kernel<S, true, false>)
                : (bz ? gemm_split_fused_kernel<S, false, true> : gemm_split_fused_kernel<S, false, false>);
  TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TKB_CUDA_TRY(ctx, launch_pdl(k, dim3((unsigned)ctx->num_sms), dim3(kFusedThreads), smem, ctx->stream, fa));
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

int64_t roundup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

}  // namespace

int tkb_gemm_split_prepare(tkb_ctx *ctx, tkb_plan *p) {
  const bool cplx = p->dtype == TKB_C128;
  int S = p->slices;
  p->slices_fixed = S > 0 ? 1 : 0;
  if (S <= 0) S = SMAX;
  if (S < 3 || S > SMAX) return tkb_set_error(ctx, TKB_ERR_UNSUPPORTED, "slices must be in 3..7");
  p->slices = S;
  size_t off = 0;
  struct SJob {
    int32_t block, op, nsrc, nchunk;
  };
  std::vector<SJob> sj;
  std::vector<GTile> tiles;
  for (size_t bi = 0; bi < p->hblocks.size(); ++bi) {
    GBlock &b = p->hblocks[bi];
    const int64_t M = cplx ? 2 * b.m : b.m;
    b.mpad = (int32_t)roundup(std::max<int64_t>(M, 1), PANEL_A);
    b.npad = (int32_t)roundup(std::max<int64_t>(b.n, 1), PANEL_B);
    // complex K: [Re | Im] halves of round_up(k, 16) positions each
    b.kpad = cplx ? (int32_t)(2 * roundup(std::max<int64_t>(b.k, 1), 16))
                  : (int32_t)roundup(std::max<int64_t>(b.k, 1), KSTAGE);
    if (b.m == 0 || b.n == 0 || b.skinny) continue;
    b.wsA = (int64_t)off;
    off += (size_t)S * b.mpad * b.kpad;
    b.wsB = (int64_t)off;
    off += (size_t)S * b.npad * b.kpad;
    off = roundup((int64_t)off, 256);
    const int kind = b.k > 0 ? 0 : 1;
    if (kind == 0) {
      // pieces of 16 real (8 complex) K values per source row
      const int32_t nchunk = cplx ? b.kpad / 2 / 8 : b.kpad / 16;
      sj.push_back({(int32_t)bi, 0, (int32_t)b.m, nchunk});
      sj.push_back({(int32_t)bi, 1, (int32_t)b.n, nchunk});
    }
    for (int64_t m0 = 0; m0 < M; m0 += PANEL_A)
      for (int64_t n0 = 0; n0 < b.n; n0 += PANEL_B) tiles.push_back({(int32_t)bi, (int32_t)m0, (int32_t)n0, kind});
  }
  // slicing tasks: as many source rows per task as keep every thread's pieces in registers
  // (kSliceKeep pieces of kSlicePlanThreads threads; at most kSliceMaxRows rows), halved while
  // there would be fewer tasks than SMs. Only the operands' own rows are sliced: padding rows of a
  // panel feed output rows and columns that are never stored.
  std::vector<SliceTask> jobs;
  if (!sj.empty()) {
    for (int div = 1;; div *= 2) {
      jobs.clear();
      for (const SJob &t : sj) {
        const int64_t rt =
            std::min<int64_t>(kSliceMaxRows, std::max<int64_t>(1, (int64_t)kSliceKeep * kSlicePlanThreads / t.nchunk));
        const int32_t r = (int32_t)std::max<int64_t>(1, rt / div);
        for (int32_t r0 = 0; r0 < t.nsrc; r0 += r) jobs.push_back({t.block, t.op, r0, std::min(r, t.nsrc - r0)});
      }
      if ((int64_t)jobs.size() >= ctx->num_sms || div >= 8) break;
    }
    // the tasks with the most pieces first
    std::vector<int32_t> nch(p->hblocks.size(), 0);
    for (const SJob &t : sj) nch[t.block] = t.nchunk;
    std::stable_sort(jobs.begin(), jobs.end(), [&](const SliceTask &x, const SliceTask &y) {
      return (int64_t)x.nrows * nch[x.block] > (int64_t)y.nrows * nch[y.block];
    });
  }
  // exponent arrays of every block in one contiguous region (rewritten by every launch)
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
  // products items of the persistent kernel (one CTA per SM). With fewer tiles than SMs the K
  // loops are cut into pieces of about `target` stages, the smallest target (≥ min_piece_steps) whose
  // item count still fits one round of the CTAs, so the longest item is as short as possible.
  std::vector<SplitTile> kt;
  int nslots = 0, npart = 0;
  {
    const int64_t nt = (int64_t)tiles.size();
    const int64_t nsm = ctx->num_sms;
    int64_t total = 0, maxnk = 1;
    for (const GTile &t : tiles)
      if (t.kind == 0) {
        total += p->hblocks[t.block].kpad / KSTAGE;
        maxnk = std::max<int64_t>(maxnk, p->hblocks[t.block].kpad / KSTAGE);
      }
    // int32 accumulators stay exact over at most (2^31 − 1)/(S·127²) K positions per item
    const int64_t maxst = std::max<int64_t>(1, (int64_t)2147483647 / ((int64_t)S * 127 * 127) / KSTAGE);
    auto pieces = [&](int64_t nk, int64_t target) {
      return (int)std::max<int64_t>(std::min<int64_t>(p->max_pieces, (nk + target - 1) / target),
                                    (nk + maxst - 1) / maxst);
    };
    int64_t target = maxnk;  // no split
    if (nt < nsm) {
      target = std::max<int64_t>(p->min_piece_steps, (total + nsm - 1) / nsm);
      for (; target < maxnk; ++target) {
        int64_t cnt = 0;
        for (const GTile &t : tiles) cnt += t.kind == 0 ? pieces(p->hblocks[t.block].kpad / KSTAGE, target) : 1;
        if (cnt <= nsm) break;
      }
    }
    for (const GTile &t : tiles) {
      const int nk = p->hblocks[t.block].kpad / KSTAGE;
      const int ks = t.kind == 0 ? pieces(nk, target) : 1;
      if (ks == 1) {
        kt.push_back({t.block, t.m0, t.n0, t.kind, 0, t.kind == 0 ? nk : 0, -1, 1, 0, 0});
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
  p->nsrows = (int64_t)jobs.size();
  cudaError_t e = cudaSuccess;
  if (!tiles.empty()) {
    e = cudaMalloc((void **)&p->stiles, tiles.size() * sizeof(GTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->stiles, tiles.data(), tiles.size() * sizeof(GTile), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !kt.empty()) {
    e = cudaMalloc(&p->kstiles, kt.size() * sizeof(SplitTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->kstiles, kt.data(), kt.size() * sizeof(SplitTile), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && nslots > 0)
    e = cudaMalloc((void **)&p->part, (size_t)npart * 64 * 128 * sizeof(double));
  // claim, finish and check counts, readiness counts, then one split-K arrival counter per split
  // tile; the block statistics; the per-block slice counts of the last launch
  const size_t nb = p->hblocks.size();
  const size_t ncnt = 3 + 2 * nb + (size_t)nslots;
  if (e == cudaSuccess) e = cudaMalloc((void **)&p->pcnt, ncnt * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(p->pcnt, 0, ncnt * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&p->bstat, std::max<size_t>(1, 4 * nb) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(p->bstat, 0, std::max<size_t>(1, 4 * nb) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void **)&p->bslices, (nb + 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(p->bslices, 0xff, (nb + 1) * sizeof(int32_t));
  if (e == cudaSuccess && !jobs.empty()) {
    e = cudaMalloc(&p->sjobs, jobs.size() * sizeof(SliceTask));
    if (e == cudaSuccess) e = cudaMemcpy(p->sjobs, jobs.data(), jobs.size() * sizeof(SliceTask), cudaMemcpyHostToDevice);
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
  if (p->dtype == TKB_C128 && ((((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15) != 0))
    return tkb_set_error(ctx, TKB_ERR_ARG, "ComplexF64 data must be 16-byte aligned");
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
