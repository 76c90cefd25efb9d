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
#include <map>
#include <mutex>
#include <numeric>

#include "tkb_internal.h"

namespace {

constexpr int PANEL_A = 128, PANEL_B = 64;   // rows per panel
constexpr int KSTAGE = 32;                   // bytes of K per stage (one tensor-core K step)
constexpr int kSmemMax = 232448;             // dynamic shared memory per CTA (227 KiB)
constexpr int kSmemTail = 2048;              // barriers and small tables after the ring
constexpr int kXchgBytes = 2 * 128 * 32 * 8;  // split tiles: this CTA's column half and the peer's
// depth of the shared-memory ring: as many stages of S slices of A and B as fit, at most 8
__host__ __device__ constexpr int ring_stages(int S) {
  return (kSmemMax - kSmemTail - kXchgBytes) / (S * (PANEL_A + PANEL_B) * KSTAGE) < 8
             ? (kSmemMax - kSmemTail - kXchgBytes) / (S * (PANEL_A + PANEL_B) * KSTAGE)
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

// byte offset of (slice 0, row r, K byte kb) in a block's slices (pr: rows per panel, 64 or
// 128); slice s is s·pr·KSTAGE bytes further
__host__ __device__ __forceinline__ int64_t slice_off(int64_t r, int64_t kb, int64_t kpad, int pr, int S) {
  const int lpr = pr == 128 ? 7 : 6;
  const int64_t panel = r >> lpr, rr = r & (pr - 1);
  const int64_t stg = kb >> 5, kk = kb & 31;
  return (panel * kpad + stg * KSTAGE) * (int64_t)(S * pr) + (rr >> 3) * 256 + (kk >> 4) * 128 + (rr & 7) * 16 +
         (kk & 15);
}

// Slicing: one task = nrows source rows of one operand of one block over the whole K range, run
// by one warp. Source rows are the rows of op(A) and the columns of op(B) (for ComplexF64 a
// complex source row of op(A) gives the real row pair 2r, 2r+1). A row is cut into pieces of LK
// consecutive K values (LK = 16 real values: one 16-byte slice store; 8 complex values: one
// 8-byte store per real row and K half). The warp's lanes form R rows × G piece groups
// (lane = g·R + r): lane (g, r) takes the pieces g, g+G, … of row r of the current R rows.
//   rows contiguous in memory (real op(A) = A, op(B) = Bᵀ; complex likewise): R ≥ 8, so every
//     load instruction reads R consecutive rows (64 bytes and more);
//   K contiguous (op(A) = Aᵀ/Aᴴ, op(B) = B): a lane reads its pieces as 16-byte vectors when the
//     row is aligned; G covers the row's pieces (R = 1 for rows of 32 pieces and more).
// Pass 1 reduces every row's largest magnitude and sum of squares (shuffles over the G lanes of
// the row) and sets the row exponent; pass 2 reads the pieces again (from L2) and writes the S
// slices. The warp then publishes its rows to the products through the readiness counts.
struct SliceTask {  // one entry per task, with every block field the task needs (one load round)
  int64_t xoff;     // element offset of source row 0 in A or B
  int64_t rs, ks;   // source row and K strides in elements
  int64_t ws_s;     // workspace byte offset of the operand's slices
  int64_t ws_e;     // workspace byte offset of the operand's row exponents
  int32_t block;
  int32_t operand;  // 0 = rows of op(A), 1 = columns of op(B)
  int32_t r0;       // first source row
  int32_t nrows;    // source rows of the task
  int32_t msrc;     // source rows of the operand
  int32_t k;        // K of the block (source values per row)
  int32_t kpad;     // padded K of the slices
  int32_t conj;     // 1: conjugate the values (op = C)
};

constexpr int kTaskPieces = 32;  // pieces per slicing task the planner aims at (one pass of a warp)

// piece groups G of a slicing warp (rows per pass R = 32 / G): the smallest power of two that
// leaves every lane one piece of a row, at most 32 (each pass of the warp is then one load
// latency for rows of up to 32 pieces, whatever the layout; rows contiguous in memory share their
// 32-byte sectors with the tasks of the neighbouring rows, which find them in L2)
__host__ __device__ __forceinline__ int slice_groups(int nchunk) {
  int g = 1;
  while (g < nchunk && g < 32) g <<= 1;
  return g;
}

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
// ks), zero beyond ksrc or for an invalid row; K-contiguous real rows (ks = 1) are read as 16-byte
// vectors where the piece is whole and aligned
template <bool CPLX, int LK>
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
  if constexpr (!CPLX) {
    if (ks == 1 && c + LK <= ksrc && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
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
// fire-and-forget maximum into global memory (no value returned, so nothing waits for it)
__device__ __forceinline__ void red_max_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;\n" ::: "memory");
}

// One slicing task run by the calling warp (every lane calls): row exponents into the
// workspace, the S slices of every row, the block statistics into bst. A lane keeps its first
// piece of a row in registers between the passes; only rows of more than G pieces are read twice
// (the second time from L2).
template <int S, bool CPLX>
__device__ __forceinline__ void slice_warp_task(const SliceTask &task, const void *Xv, int8_t *ws,
                                                unsigned long long *bst) {
  using T = typename SrcVal<CPLX>::T;
  constexpr int LK = CPLX ? 8 : 16;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int op = task.operand;
  const int64_t rs = task.rs, ks = task.ks;
  const int64_t kfull = CPLX ? task.kpad / 2 : task.kpad;
  const int nchunk = (int)(kfull / LK);
  const int G = slice_groups(nchunk), R = 32 / G;
  const int gq = lane / R, rr = lane - gq * R;
  const bool conj = task.conj != 0;
  const T *X = reinterpret_cast<const T *>(Xv);
  int8_t *base = ws + task.ws_s;
  int32_t *ex = reinterpret_cast<int32_t *>(ws + task.ws_e);
  unsigned ebm = 0u;  // largest biased exponent of the task's nonzero rows
  double nrm = 0.0;   // largest 2-norm of the task's rows
#pragma unroll 1
  for (int rb = 0; rb < task.nrows; rb += R) {
    const int64_t r = task.r0 + rb + rr;
    const bool rv = rb + rr < task.nrows && r < task.msrc;
    const int64_t rowbase = task.xoff + r * rs;
    // pass 1: the lane's first piece (kept in registers), then any further pieces; lanes past the
    // row's last piece (gq ≥ nchunk) hold zeros and store nothing
    const bool has = rv && gq < nchunk;
    T v0[LK];
    load_piece<CPLX, LK>(X, rowbase, ks, (int64_t)gq * LK, task.k, has, v0);
    double m = 0.0, s2 = 0.0;
#pragma unroll
    for (int l = 0; l < LK; ++l) {
      m = fmax(m, absmax(v0[l]));
      s2 += sq_of(v0[l]);
    }
#pragma unroll 1
    for (int c = gq + G; c < nchunk; c += G) {
      T w[LK];
      load_piece<CPLX, LK>(X, rowbase, ks, (int64_t)c * LK, task.k, rv, w);
#pragma unroll
      for (int l = 0; l < LK; ++l) {
        m = fmax(m, absmax(w[l]));
        s2 += sq_of(w[l]);
      }
    }
#pragma unroll 1
    for (int o = R; o < 32; o <<= 1) {
      m = fmax(m, __shfl_xor_sync(full, m, o));
      s2 += __shfl_xor_sync(full, s2, o);
    }
    const int e = row_exponent<S>(m);
    if (rv && gq == 0) {
      if (CPLX && op == 0) {
        ex[2 * r] = e;
        ex[2 * r + 1] = e;
      } else {
        ex[r] = e;
      }
    }
    if (rv && m > 0.0) {
      ebm = max(ebm, (unsigned)(e + kExpBias));
      nrm = fmax(nrm, sqrt(s2));
    }
    // pass 2: the slices of the kept piece, then of the further pieces (read again, from L2)
    if (has) store_piece<S, CPLX, LK>(v0, op, conj, r, (int64_t)gq * LK, kfull, task.kpad, base, e);
#pragma unroll 1
    for (int c = gq + G; c < nchunk; c += G) {
      T w[LK];
      load_piece<CPLX, LK>(X, rowbase, ks, (int64_t)c * LK, task.k, rv, w);
      if (rv) store_piece<S, CPLX, LK>(w, op, conj, r, (int64_t)c * LK, kfull, task.kpad, base, e);
    }
  }
  ebm = __reduce_max_sync(full, ebm);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nrm = fmax(nrm, __shfl_xor_sync(full, nrm, o));
  if (lane == 0 && ebm != 0u) {
    red_max_u64(&bst[4 * task.block + op], (unsigned long long)ebm);
    red_max_u64(&bst[4 * task.block + 2 + op], (unsigned long long)__double_as_longlong(nrm));
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

// Timeline build (compiled with -DTKB_TIMELINE into a separate library): per CTA, global-timer
// stamps (ns) at fixed points of the fused kernel, counts, and wait/work time sums, read back
// with tkb_timeline_read. The default build compiles every stamp away.
#ifdef TKB_TIMELINE
constexpr int kTlCtas = 256, kTlSlots = 32;
__device__ unsigned long long tkb_tl[kTlCtas * kTlSlots];
#define TL_AT(k) (tkb_tl[blockIdx.x * kTlSlots + (k)])
#define TL_STAMP(k)                                 \
  do {                                              \
    if (blockIdx.x < kTlCtas) TL_AT(k) = globaltimer_ns(); \
  } while (0)
#define TL_ADD(k, v)                                                          \
  do {                                                                        \
    if (blockIdx.x < kTlCtas) atomicAdd(&TL_AT(k), (unsigned long long)(v)); \
  } while (0)
#define TL_MAX(k, v)                                                          \
  do {                                                                        \
    if (blockIdx.x < kTlCtas) atomicMax(&TL_AT(k), (unsigned long long)(v)); \
  } while (0)
#define TL_NOW() globaltimer_ns()
#else
#define TL_MAX(k, v) ((void)0)
#define TL_STAMP(k) ((void)0)
#define TL_ADD(k, v) ((void)0)
#define TL_NOW() 0ull
#endif
// one test of a phase parity (the hardware may suspend the thread for a while before it answers)
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait on a phase parity: false once 2 s of wall time have passed. A phase that has
// completed costs one test; the clock is read only after the first test fails, then every 64.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  if (mbar_try(addr, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t n = 1;; ++n) {
    if (mbar_try(addr, parity)) return true;
    if ((n & 63u) == 0 && globaltimer_ns() - t0 > 2000000000ull) return false;
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
  const unsigned long long ea = __ldcg(&bst[4 * block]), eb = __ldcg(&bst[4 * block + 1]);
  if (ea == 0ull || eb == 0ull) return SM;  // an operand of the block is zero: so are its products
  const double na = __longlong_as_double((long long)__ldcg(&bst[4 * block + 2]));
  const double nb = __longlong_as_double((long long)__ldcg(&bst[4 * block + 3]));
  const double k = (double)kpad;
  const double cmax = 4.5 * na * nb / sqrt(k);
  const int e = (int)ea + (int)eb - 2 * kExpBias;
  for (int s = 3; s <= SM; ++s) {
    const double est = kGuardSigma * sqrt((double)s * k) * scale2(1.0, e - 7 * s);
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
// (The four warps of one column half, called alone with n0 moved by 32·half and warp − 4·half,
// compute that half.)
// Real: tile rows m0 .. m0+127, warp (w mod 4, w / 4) takes 32 rows × 32 columns. Complex: the
// tile's real row pairs are complex rows m0/2 .. m0/2+63; a warp takes 16 complex rows × 32
// columns, four real DMMA per complex product.
template <bool CPLX>
__device__ __noinline__ void fp64_tile(const GBlock &b, int64_t m0, int64_t n0, const void *A, const void *B,
                                       double *C, CDbl alpha, CDbl beta, bool bz, int warp, int lane) {
  if (n0 >= b.n) return;
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
  int *cnt;                 // [1] finished product CTAs, [2] tiles recomputed in FP64,
                            // [4 + block] source rows sliced (both operands),
                            // [4 + nblocks + block] the block's slice count + 1 (0: not yet sliced)
  unsigned long long *bst;  // 4 per block: statistics of the slicing
  int *slices_out;          // per block: the slice count of the last launch (0 = FP64, −1 = no
                            // products), then the number of tiles the check sent to FP64
  double *part;             // split-K partial tiles, [col][row] per piece, then one hold tile per CTA
  int hold0;                // index of CTA 0's hold tile in part
  int *err;
  CDbl alpha, beta;
  int nstasks, nitems, nblocks;
  int nctasks;              // the first nctasks slicing tasks are staged CTA tasks
  int fixed;                // 1: the caller fixed the slice count (every block uses S, no check)
};

// bounded mbarrier wait that also gives up when the CTA aborts (a completed phase costs one test)
__device__ __forceinline__ bool mbar_wait_abortable(uint64_t *bar, uint32_t parity, const volatile int *abort) {
  const uint32_t addr = smem_u32(bar);
  if (mbar_try(addr, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t n = 1;; ++n) {
    if (mbar_try(addr, parity)) return true;
    if (*abort) return false;
    if ((n & 63u) == 0 && globaltimer_ns() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// bounded wait until *p ≥ target (acquire at GPU scope); false once 2 s have passed or the CTA
// aborts (a count already reached costs one load)
__device__ __forceinline__ bool wait_at_least(const int *p, int target, const volatile int *abort) {
  if (ld_acquire(p) >= target) return true;
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    __nanosleep(64);
    if (ld_acquire(p) >= target) return true;
    if (*abort || globaltimer_ns() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// ---- the two CTAs of a cluster (split tiles exchange column halves) ---------------------------
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
// the shared::cluster address of this CTA's shared-memory address in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_peer_f64(uint32_t addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;\n" ::"r"(addr), "d"(v) : "memory");
}
// arrive on an mbarrier of the peer CTA, releasing this thread's earlier writes at cluster scope
__device__ __forceinline__ void mbar_arrive_peer(uint32_t addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(addr) : "memory");
}
__device__ __forceinline__ void fence_cluster() { asm volatile("fence.acq_rel.cluster;\n" ::: "memory"); }
// every thread of both CTAs (release / acquire at cluster scope)
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// bounded wait on a phase parity with acquire at cluster scope (arrivals of the peer CTA);
// false once 2 s have passed or the CTA aborts
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *bar, uint32_t parity, const volatile int *abort) {
  const uint32_t addr = smem_u32(bar);
  auto test = [&]() {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
  };
  if (test()) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t n = 1;; ++n) {
    if (test()) return true;
    if (*abort) return false;
    if ((n & 63u) == 0 && globaltimer_ns() - t0 > 2000000000ull) return false;
  }
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

// exact int32 → double without a conversion instruction: the bits 0x43300000:(x ^ 2^31) are the
// double 2^52 + 2^31 + x, from which 2^52 + 2^31 is subtracted exactly
__device__ __forceinline__ double i32_to_f64(uint32_t x) {
  return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 4503601774854144.0;
}
// the first Sb int32 diagonals of one output combined in FP64, times 2^(7(Sb+1)): Horner in base
// 128 (every diagonal converts exactly; once the partial sum passes 2^53 each fused multiply-add
// rounds, a relative error of a few 2^-53 of the diagonals' scale, far below the truncation)
template <int S, int W>
__device__ __forceinline__ double recombine_value(const uint32_t (&r)[S][W], int q, int Sb) {
  double acc = i32_to_f64(r[0][q]);
#pragma unroll
  for (int d = 1; d < S; ++d)
    if (d < Sb) acc = fma(acc, 128.0, i32_to_f64(r[d][q]));
  return acc;
}

// the α/β update and store of 8 values of one row (columns j0 .. j0+7); real or complex rows
// (complex: every lane takes part, the partner row comes by shuffle)
template <bool CPLX>
__device__ __forceinline__ void store_group(const double (&v)[8], int64_t i, int64_t j0, const GBlock &b, double *C,
                                            CDbl alpha, CDbl beta, bool bz) {
  if constexpr (!CPLX) {
    const int nj = (int)min((int64_t)8, b.n - j0);
    if (i >= b.m || nj <= 0) return;
    double *pc = C + b.offC + i + j0 * b.ldc;
    double old[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) old[q] = (!bz && q < nj) ? pc[q * b.ldc] : 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (q < nj) pc[q * b.ldc] = bz ? alpha.x * v[q] : fma(beta.x, old[q], alpha.x * v[q]);
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) store_out(v[q], i, j0 + q, b, 1, C, alpha, beta, bz, 1);
  }
}

template <int S, bool CPLX, bool BZ>
__global__ void __launch_bounds__(kFusedThreads, 1) gemm_split_fused_kernel(const FusedArgs args) {
  constexpr uint32_t A_BYTES = S * PANEL_A * KSTAGE, B_BYTES = S * PANEL_B * KSTAGE;
  constexpr uint32_t A_SLICE = PANEL_A * KSTAGE, B_SLICE = PANEL_B * KSTAGE;
  constexpr uint32_t STAGE = A_BYTES + B_BYTES;
  constexpr int NSTAGE = ring_stages(S);
  extern __shared__ __align__(1024) unsigned char smem[];
  // split tiles: this CTA's column half of its own piece (xo) and the peer's piece for it (xr),
  // [column][row] of 32 × 128
  double *xo = reinterpret_cast<double *>(smem + NSTAGE * STAGE);
  double *xr = xo + 32 * 128;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * STAGE + kXchgBytes);
  uint64_t *empty = full + NSTAGE;
  uint64_t *acc_full = full + 2 * NSTAGE;
  uint64_t *acc_empty = acc_full + 1;
  uint64_t *drain = acc_full + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_full + 3);
  volatile int *abort = reinterpret_cast<int *>(acc_full + 4);
  uint64_t *xfull = acc_full + 5;   // xr holds the peer's half (4 arrivals of the peer's warps)
  uint64_t *xempty = acc_full + 6;  // the peer has read this CTA's half out of its xr (4 arrivals)
  // tile check: per epilogue warp, largest |C|, row exponent and column exponent (two buffers)
  double *gmax = reinterpret_cast<double *>(acc_full + 8);    // [2][kEpiWarps]
  int *gexp = reinterpret_cast<int *>(gmax + 2 * kEpiWarps);        // [2][kEpiWarps][2]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const FusedArgs &g = args;
  // the cluster of two CTAs takes the item pairs cl, cl + ncl, …; rank r the pair's item r
  const int rank = (int)cluster_rank(), peer = rank ^ 1;
  const int cl = (int)blockIdx.x >> 1, ncl = (int)gridDim.x >> 1;
  auto item_of = [&](int k) { return 2 * (cl + k * ncl) + rank; };
  if (tid == 0) TL_STAMP(0);

  if (tid == 0) {
#pragma unroll
    for (int st = 0; st < NSTAGE; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kEpiWarps);
    mbar_init(drain, 1);
    mbar_init(xfull, kEpiWarps / 2);
    mbar_init(xempty, kEpiWarps / 2);
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
  cluster_sync_all();  // the peer's barriers are initialised before any arrival on them
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // the item table and block descriptors are plan constants: the first item and its block are
  // brought into L1 while the slicing launch finishes
  if (lane == 0 && item_of(0) < g.nitems) {
    const SplitTile it0 = g.items[item_of(0)];
    const char *pb = reinterpret_cast<const char *>(g.blocks + it0.block);
    for (int o = 0; o < (int)sizeof(GBlock); o += 64) asm volatile("prefetch.L1 [%0];\n" ::"l"(pb + o));
  }
  // No wait for the slicing launch to finish: every role waits for the readiness counts of its
  // item's block instead (the slicing launch publishes each task's rows). This launch starts
  // only once every CTA of the slicing launch runs (which in turn began after the earlier kernels
  // of the stream had finished), so the counts always complete, and C and the FP64 operands are
  // final.
  int *ready = g.cnt + 4;  // [block]: source rows sliced (both operands); [nblocks + block]: slice count + 1
  if (tid == 0) TL_STAMP(1);

  // ---- products ------------------------------------------------------------------
  // a block's slice count (0: the block runs in FP64) from the statistics of the slicing launch
  // bounded wait until both operands of a block are sliced; the slicing task that completes the
  // block publishes its slice count as sb + 1 (acquire: the slices, exponents and statistics of
  // the block are visible after it). −1 on timeout or abort.
  auto sliced = [&](int block) -> int {
    return wait_at_least(&ready[g.nblocks + block], 1, abort) ? ld_acquire(&ready[g.nblocks + block]) - 1 : -1;
  };
  if (warp == kProducerWarp) {
    if (lane == 0) {
      int issued = 0, landed = 0;  // stages issued / known to have landed (for the final drain)
      int gs = 0;                  // ring stage counter over all items of this CTA
      for (int k = 0, ii = item_of(0); ii < g.nitems && !*abort; ii = item_of(++k)) {
        const SplitTile it = g.items[ii];
        if (it.kind != 0) continue;
        const GBlock b = g.blocks[it.block];
        const int sb = sliced(it.block);
        if (sb < 0) {
          atomicExch(g.err, 3);
          *abort = 1;
          break;
        }
        if (issued == 0) TL_STAMP(7);
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
      TL_STAMP(8);
      // every bulk copy must land before the CTA can exit (bounded)
      for (int k = landed; k < issued; ++k) mbar_wait(&full[k % NSTAGE], (k / NSTAGE) & 1);
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      int gs = 0, li = 0;
      bool ok = true;
      for (int k = 0, ii = item_of(0); ii < g.nitems && ok && !*abort; ii = item_of(++k)) {
        const SplitTile it = g.items[ii];
        if (it.kind != 0) continue;
        const int sb = sliced(it.block);
        if (sb < 0) {
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
          if (li == 0 && kt == it.kb) {
            TL_STAMP(2);
            TL_ADD(15, it.ke - it.kb);
          }
          tc_fence_after();
          const uint32_t a0 = ring0 + st * STAGE, b0 = a0 + A_BYTES;
          // the products (s, t), (s, t+1), … share the A slice s and land in the adjacent
          // diagonals s+t, …; up to four B slices (back to back in the stage) form one N ≤ 256
          // operand
          if (S == 7 && sb == 7) {
            // 7 slices: the ten instructions in an order where neighbours mostly write disjoint
            // diagonals (each A slice has one instruction that reaches diagonal 6, so three
            // neighbouring pairs at least overlap); consecutive MMAs into overlapping accumulator
            // columns measured 12–15 % slower per K stage. The two s = 0 instructions come first:
            // at the item's first stage they start the seven diagonals.
            constexpr int ord_s[10] = {0, 0, 1, 1, 2, 2, 6, 3, 5, 4};
            constexpr int ord_t[10] = {0, 4, 4, 0, 4, 0, 0, 0, 0, 0};
#pragma unroll 1
            for (int q = 0; q < 10; ++q) {
              const int s = ord_s[q], tt = ord_t[q];
              const int nsl = (7 - s - tt) < kMaxSlicesPerMma ? (7 - s - tt) : kMaxSlicesPerMma;
              umma_i8(tmem + (uint32_t)((s + tt) * 64), umma_desc(a0 + s * A_SLICE, 128, 256),
                      umma_desc(b0 + tt * B_SLICE, 128, 256), idesc_i8(64u * (uint32_t)nsl),
                      (kt > it.kb || s > 0) ? 1u : 0u);
            }
          } else {
#pragma unroll 1
          for (int s = 0; s < S; ++s) {
            if (s < sb) {
              const uint64_t ad = umma_desc(a0 + s * A_SLICE, 128, 256);
#pragma unroll 1
              for (int tt = 0; tt < S - s; tt += kMaxSlicesPerMma) {
                if (tt < sb - s) {
                  const int nsl = (sb - s - tt) < kMaxSlicesPerMma ? (sb - s - tt) : kMaxSlicesPerMma;
                  umma_i8(tmem + (uint32_t)((s + tt) * 64), ad, umma_desc(b0 + tt * B_SLICE, 128, 256),
                          idesc_i8(64u * (uint32_t)nsl), (kt > it.kb || s > 0) ? 1u : 0u);
                }
              }
            }
          }
          }
          umma_commit(&empty[st]);
        }
        if (!ok) break;
        umma_commit(acc_full);
        if (li == 0) TL_STAMP(9);
        ++li;
      }
      TL_STAMP(10);
      // every MMA issued by this thread completes before TMEM is released (bounded)
      umma_commit(drain);
      mbar_wait(drain, 0);
    }
    __syncwarp();
  } else {
    // epilogue warps: warp w owns TMEM lanes 32(w mod 4) .. +31 (its rows) and the 32 columns
    // 32·half .. +31, half = w / 4. In a split tile (two K pieces on the two CTAs of the cluster)
    // CTA r keeps column half r: its warps of half r put their values into xo, the warps of the
    // other half send theirs into the peer's xr; the warps of half r then add xo and xr, check and
    // store that half.
    const int quarter = warp & 3, half = warp >> 2;
    const int row = 32 * quarter + lane;
    const bool keeper = half == rank;
    constexpr bool bz = BZ;
    const uint32_t xr_peer = peer_addr(smem_u32(xr), (uint32_t)peer);
    const uint32_t xempty_peer = peer_addr(smem_u32(xempty), (uint32_t)peer);
    const uint32_t xfull_peer = peer_addr(smem_u32(xfull), (uint32_t)peer);
    int li = 0, gi = 0, ns = 0;  // items with products, checked tiles, exchanged split tiles
    for (int k = 0, ii = item_of(0); ii < g.nitems; ii = item_of(++k)) {
      const SplitTile it = g.items[ii];
      if (it.kind == 2) continue;  // the empty half of a pair
      const GBlock b = g.blocks[it.block];
      const int64_t Mreal = CPLX ? 2 * b.m : b.m;
      const int64_t i = it.m0 + row;
      const bool prod = it.kind == 0;
      bool stop = *abort != 0;
      int sb = 0;
      if (prod && !stop) {
        // lane 0 acquires the block's slice count; __syncwarp orders the other lanes' reads of the
        // exponents after that acquire
        if (lane == 0) sb = sliced(it.block);
        __syncwarp();
        sb = __shfl_sync(0xffffffffu, sb, 0);
        stop = sb < 0;
        if (stop) sb = 0;
      }
      const bool mma = prod && sb > 0;  // the tile's products ran on the tensor cores
      // the row exponent and the exponent of this lane's column, read before the products finish
      const int32_t *eA = reinterpret_cast<const int32_t *>(g.ws + b.wsEA);
      const int32_t *eB = reinterpret_cast<const int32_t *>(g.ws + b.wsEB);
      const bool rok = i < Mreal;
      const int64_t jl = it.n0 + 32 * half + lane;
      const bool cok = jl < b.n;
      const int eA_i = mma && rok ? eA[i] : -1100;
      const int eB_j = mma && cok ? eB[jl] : -1100;
      [[maybe_unused]] const unsigned long long ta = TL_NOW();
      if (mma && !stop) stop = !mbar_wait_abortable(acc_full, li & 1, abort);
      if (tid == 0) {
        TL_ADD(21, TL_NOW() - ta);
        if (li == 0 && mma) TL_STAMP(11);
        TL_ADD(18, 1);
      }
      [[maybe_unused]] const unsigned long long tr = TL_NOW();
      if (epi_any(stop)) {  // every epilogue warp leaves the loop here, together
        if (tid == 0) {
          atomicExch(g.err, 2);
          *abort = 1;
        }
        break;
      }
      if (prod && !mma) {
        // FP64 block: the first piece computes the whole tile over the full K range
        if (it.sid == 0) fp64_tile<CPLX>(b, it.m0, it.n0, g.A, g.B, g.C, g.alpha, g.beta, bz, warp, lane);
        continue;
      }
      const bool split = it.nsplit > 1;
      // direct: β = 0 and one piece, so the values go to C as they are recombined (a tile the
      // check sends to FP64 is overwritten). β ≠ 0, one piece: they wait in the CTA's hold tile
      // ([col][row], global) until the check has passed.
      const bool direct = BZ && !split;
      double *scr = g.part + (int64_t)(g.hold0 + (int)blockIdx.x) * (64 * 128);
      double vmax = 0.0;    // largest |C| of the thread's values
      int ei = 0, ejm = 0;  // the thread's row exponent, the largest column exponent of its columns
      if (mma) {
        tc_fence_after();
        // rows past the block (and columns, below) get exponent −1100 and scale 0: their values
        // become zero and are never stored
        ei = rok ? max(eA_i, -1100) : -1100;
        // the row scale carries the recombination's 2^(−7(sb+1))
        const int eis = ei - 7 * (sb + 1);
        const double rscale = (eis >= -1022 && eis <= 1023) ? pow2i(eis) : 0.0;
        // lane l holds the exponent and scale of the warp's column 32·half + l (shared by shuffles)
        const int ej = cok ? max(eB_j, -1100) : -1100;
        const double cs = (ej >= -1022 && ej <= 1023) ? pow2i(ej) : 0.0;
        ejm = ej;
        // the exact (ldexp) scaling only where a real row's or column's 2^e is not a normal double
        const bool slow = __any_sync(0xffffffffu, (rok && rscale == 0.0) || (cok && cs == 0.0));
        // a sending warp may overwrite the peer's xr once the peer has read the previous split tile
        if (split && !keeper && ns > 0 && !mbar_wait_cluster(xempty, (ns - 1) & 1, abort)) stop = true;
        // the warp's 32 columns, 8 at a time (a runtime loop: the code stays small); after the
        // last group's loads the accumulators go back to the MMA warp
#pragma unroll 1
        for (int g8 = 0; g8 < 4; ++g8) {
          const int c0 = 32 * half + 8 * g8;
          double w[8];
          {
            uint32_t r[S][8];
#pragma unroll
            for (int d = 0; d < S; ++d)
              if (d < sb) tmem_ld8_issue(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(d * 64 + c0), r[d]);
#pragma unroll
            for (int d = 0; d < S; ++d)
              if (d < sb) tmem_ld_wait8(r[d]);
            if (g8 == 3) {
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(acc_empty);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) w[q] = recombine_value<S, 8>(r, q, sb);
          }
          if (!slow) {
#pragma unroll
            for (int q = 0; q < 8; ++q) w[q] = w[q] * rscale * __shfl_sync(0xffffffffu, cs, 8 * g8 + q);
          } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) w[q] = scale2(w[q], eis + __shfl_sync(0xffffffffu, ej, 8 * g8 + q));
          }
#pragma unroll
          for (int q = 0; q < 8; ++q) vmax = fmax(vmax, fabs(w[q]));
          if (direct) {
            store_group<CPLX>(w, i, it.n0 + c0, b, g.C, g.alpha, g.beta, true);
          } else if (!split) {
#pragma unroll
            for (int q = 0; q < 8; ++q) __stcg(&scr[(c0 + q) * 128 + row], w[q]);
          } else if (keeper) {
#pragma unroll
            for (int q = 0; q < 8; ++q) xo[(8 * g8 + q) * 128 + row] = w[q];
          } else if (!stop) {
#pragma unroll
            for (int q = 0; q < 8; ++q) st_peer_f64(xr_peer + (uint32_t)(((8 * g8 + q) * 128 + row) * 8), w[q]);
          }
          if (tid == 0 && li == 0 && g8 == 0) TL_STAMP(13);
        }
        if (tid == 0) {
          if (li == 0) TL_STAMP(12);
          TL_ADD(22, TL_NOW() - tr);
        }
        ++li;
      }
      if (!mma) {  // β-scale only (k = 0)
#pragma unroll 1
        for (int g8 = 0; g8 < 4; ++g8) {
          const double w[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
          store_group<CPLX>(w, i, it.n0 + 32 * half + 8 * g8, b, g.C, g.alpha, g.beta, bz);
        }
        continue;
      }
      [[maybe_unused]] const unsigned long long ts = TL_NOW();
      if (split) {
        // sending warps: their values are in the peer's xr; keeping warps: wait for the peer's
        // half, add it to their own (two terms: the order does not matter), then free xr
        if (!keeper) {
          fence_cluster();
          __syncwarp();
          if (lane == 0) mbar_arrive_peer(xfull_peer);
          vmax = 0.0;
          ei = -1100;
          ejm = -1100;
        } else {
          if (!mbar_wait_cluster(xfull, ns & 1, abort)) stop = true;
          vmax = 0.0;
#pragma unroll 4
          for (int q = 0; q < 32; ++q) {
            const double v = xo[q * 128 + row] + xr[q * 128 + row];
            xo[q * 128 + row] = v;
            vmax = fmax(vmax, fabs(v));
          }
          fence_cluster();
          __syncwarp();
          if (lane == 0) mbar_arrive_peer(xempty_peer);
        }
        ++ns;
        if (epi_any(stop)) {
          if (tid == 0) {
            atomicExch(g.err, 2);
            *abort = 1;
          }
          break;
        }
        if (tid == 0) TL_ADD(19, 1);
      }
      if (tid == 0) TL_ADD(23, TL_NOW() - ts);
      // tile check (a split tile: this CTA's column half): largest |C| and exponents against
      // the error estimate
      [[maybe_unused]] const unsigned long long tg = TL_NOW();
      double vm = vmax;
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
      const double est = kGuardSigma * sqrt((double)sb * (double)b.kpad) * scale2(1.0, te + tf - 7 * sb);
      if (!g.fixed && est > kSliceTol * tmax) {  // uniform over the epilogue warps
        if (tid == 0) atomicAdd(&g.cnt[2], 1);
        if (direct) epi_sync();  // every approximate value of the tile is stored before the overwrite
        if (!split) {
          fp64_tile<CPLX>(b, it.m0, it.n0, g.A, g.B, g.C, g.alpha, g.beta, bz, warp, lane);
        } else if (keeper) {  // this CTA's column half
          fp64_tile<CPLX>(b, it.m0, it.n0 + 32 * rank, g.A, g.B, g.C, g.alpha, g.beta, bz, warp - 4 * rank, lane);
        }
        continue;
      }
      if (split) {
        if (keeper) {
#pragma unroll 1
          for (int g8 = 0; g8 < 4; ++g8) {
            double w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) w[q] = xo[(8 * g8 + q) * 128 + row];
            store_group<CPLX>(w, i, it.n0 + 32 * half + 8 * g8, b, g.C, g.alpha, g.beta, bz);
          }
        }
      } else if (!direct) {
        // the checked values from the hold tile (written by this thread) to C
#pragma unroll 1
        for (int g8 = 0; g8 < 4; ++g8) {
          const int c0 = 32 * half + 8 * g8;
          double w[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) w[q] = __ldcg(&scr[(c0 + q) * 128 + row]);
          store_group<CPLX>(w, i, it.n0 + c0, b, g.C, g.alpha, g.beta, bz);
        }
      }
      if (tid == 0) TL_ADD(24, TL_NOW() - tg);
    }
    if (tid == 0) TL_STAMP(16);
  }

  // ---- teardown ----------------------------------------------------------------------------
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // no CTA leaves while its peer may still reach its shared memory
  if (tid == 0) TL_STAMP(17);
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
  }
  if (warp == 0) {
    // the last CTA out records the launch's slice counts and checks and clears the statistics and
    // counts for the next launch (its first warp, one block per lane)
    int last = 0;
    if (lane == 0) {
      __threadfence();
      last = atomicAdd(&g.cnt[1], 1) == (int)gridDim.x - 1;
    }
    if (__shfl_sync(0xffffffffu, last, 0)) {
      __threadfence();
      for (int q = lane; q < g.nblocks; q += 32) {
        const GBlock &b = g.blocks[q];
        const int f = ready[g.nblocks + q];
        g.slices_out[q] = (b.m > 0 && b.n > 0 && b.k > 0 && !b.skinny && f > 0) ? f - 1 : -1;
      }
      __syncwarp();
      for (int q = lane; q < 4 * g.nblocks; q += 32) g.bst[q] = 0ull;
      for (int q = lane; q < 2 * g.nblocks; q += 32) ready[q] = 0;
      if (lane == 0) {
        g.slices_out[g.nblocks] = g.cnt[2];
        g.cnt[2] = 0;
        __threadfence();
        g.cnt[1] = 0;
      }
    }
  }
}

// Staged slicing task, run by the whole CTA (every thread calls): nrows whole rows of one operand
// are copied into shared memory with cp.async (consecutive threads take consecutive addresses:
// along the rows when the rows are contiguous in memory, along K otherwise), so a task costs one
// memory round trip. Row maxima and sums of squares then come from shared memory (one warp per
// row), and every thread slices pieces of 16 real (8 complex) K values out of it. A stage row
// holds kfull values plus one padding value per piece (fewer bank conflicts between pieces).
constexpr int kStageBytes = 48 * 1024;  // shared memory of one staged task
constexpr int kStagedRowsMax = 64;      // rows of one staged task
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_u32(dst)), "l"(src), "n"(sizeof(T))
               : "memory");
}
template <int S, bool CPLX, int NT>
__device__ __forceinline__ void slice_staged(const SliceTask &task, const void *Xv, int8_t *ws, unsigned long long *bst,
                                             void *stage_v, int *rexp, unsigned long long *wstat) {
  using T = typename SrcVal<CPLX>::T;
  constexpr int LK = CPLX ? 8 : 16;
  constexpr int NW = NT / 32;
  const unsigned full = 0xffffffffu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int op = task.operand;
  const int64_t kfull = CPLX ? task.kpad / 2 : task.kpad;
  const int nchunk = (int)(kfull / LK);
  const int stride = (int)(kfull + kfull / LK);  // stage row length in elements (with padding)
  const int nrows = task.nrows;
  const bool rowc = task.rs == 1;
  T *stage = reinterpret_cast<T *>(stage_v);
  const T *X = reinterpret_cast<const T *>(Xv);
  const T z = zero_of(T{});
  // 1. copy the rows in (zeros past k and for rows past the operand)
  const int total = nrows * (int)kfull;
  // element q = tid, tid + NT, … as (r, c): the fast index (r for row-contiguous, c otherwise)
  // steps by NT mod fast with a carry into the slow one (no division per element)
  const int fast = rowc ? nrows : (int)kfull;
  const int fstep = NT % fast, sstep = NT / fast;
  int fi = tid % fast, si = tid / fast;
#pragma unroll 1
  for (int q = tid; q < total; q += NT) {
    const int r = rowc ? fi : si, c = rowc ? si : fi;
    fi += fstep;
    si += sstep;
    if (fi >= fast) {
      fi -= fast;
      ++si;
    }
    T *dst = stage + r * stride + c + c / LK;
    const int64_t rr = task.r0 + r;
    if (c < task.k && rr < task.msrc) cp_async_elem(dst, X + task.xoff + rr * task.rs + (int64_t)c * task.ks);
    else *dst = z;
  }
  asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (tid == 0) TL_STAMP(3);
  // 2. row maxima, sums of squares, exponents: eight lanes per row, four rows per warp at a time
  unsigned ebm = 0u;
  double nrm = 0.0;
  int32_t *ex = reinterpret_cast<int32_t *>(ws + task.ws_e);
  const int sub = lane >> 3, l8 = lane & 7;
#pragma unroll 1
  for (int r0 = 4 * warp; r0 < nrows; r0 += 4 * NW) {
    const int r = r0 + sub;
    double m = 0.0, s2 = 0.0;
    if (r < nrows) {
      const T *row = stage + r * stride;
#pragma unroll 4
      for (int c = l8; c < (int)kfull; c += 8) {
        const T v = row[c + c / LK];
        m = fmax(m, absmax(v));
        s2 += sq_of(v);
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      m = fmax(m, __shfl_xor_sync(full, m, o));
      s2 += __shfl_xor_sync(full, s2, o);
    }
    if (r >= nrows) continue;
    const int e = row_exponent<S>(m);
    const int64_t rr = task.r0 + r;
    if (l8 == 0) {
      rexp[r] = e;
      if (rr < task.msrc) {
        if (CPLX && op == 0) {
          ex[2 * rr] = e;
          ex[2 * rr + 1] = e;
        } else {
          ex[rr] = e;
        }
      }
    }
    if (rr < task.msrc && m > 0.0) {
      ebm = max(ebm, (unsigned)(e + kExpBias));
      nrm = fmax(nrm, sqrt(s2));
    }
  }
  // the task's block statistics: one value per warp into shared memory, one reduction per task
  // into the block statistics after the slices (the global reductions of many CTAs onto a few
  // addresses stay out of the way of the loads and stores)
  ebm = __reduce_max_sync(full, ebm);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nrm = fmax(nrm, __shfl_xor_sync(full, nrm, o));
  if (lane == 0) {
    wstat[warp] = ebm;
    wstat[NW + warp] = (unsigned long long)__double_as_longlong(nrm);
  }
  __syncthreads();
  if (tid == 0) TL_STAMP(4);
  // 3. the slices of every piece (row, p)
  int8_t *base = ws + task.ws_s;
  const int npieces = nrows * nchunk;
  const int pstep = NT % nchunk, rstep = NT / nchunk;
  int p = tid % nchunk, r = tid / nchunk;
#pragma unroll 1
  for (int q = tid; q < npieces; q += NT) {
    const int pr = p, rr0 = r;
    p += pstep;
    r += rstep;
    if (p >= nchunk) {
      p -= nchunk;
      ++r;
    }
    const int64_t rr = task.r0 + rr0;
    if (rr >= task.msrc) continue;
    const T *src = stage + rr0 * stride + pr * (LK + 1);
    T v[LK];
#pragma unroll
    for (int l = 0; l < LK; ++l) v[l] = src[l];
    store_piece<S, CPLX, LK>(v, op, task.conj != 0, rr, (int64_t)pr * LK, kfull, task.kpad, base, rexp[rr0]);
  }
  if (tid == 0) {
    unsigned long long e8 = 0ull, n8 = 0ull;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      e8 = max(e8, wstat[w]);
      n8 = max(n8, wstat[NW + w]);  // bits of non-negative doubles order like their values
    }
    if (e8 != 0ull) {
      red_max_u64(&bst[4 * task.block + op], e8);
      red_max_u64(&bst[4 * task.block + 2 + op], n8);
    }
  }
  __syncthreads();  // the stage, rexp and wstat are rewritten by the next task
  if (tid == 0) TL_STAMP(5);
}

// The slicing launch: the staged CTA tasks (the first nctasks) go to the CTAs in turn, then warp w
// of the grid takes the warp tasks w, w + W, … (W warps); each list is sorted largest first. Every
// task publishes its rows on the readiness count of its (block, operand). The launch lets the
// products launch start as soon as all its CTAs run; the products wait for the counts of their
// blocks, not for this launch to finish.
// Called by one thread once a task's slices, exponents and statistics are written (and fenced
// for the async proxy): adds the task's rows to its block's count; the task that completes the
// block (both operands) sets the block's slice count from the statistics and publishes it as
// slice count + 1 (release), which the products launch waits for.
template <int S>
__device__ __forceinline__ void publish_rows(const FusedArgs &g, const SliceTask &task) {
  const GBlock &b = g.blocks[task.block];
  // one acquire-release add: releases this task's writes (the CTA's, ordered by the barrier before
  // the call) and, for the task that completes the block, acquires every other task's statistics
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;\n"
               : "=r"(old)
               : "l"(&g.cnt[4 + task.block]), "r"(task.nrows)
               : "memory");
  if (old + task.nrows == (int)(b.m + b.n)) {
    const int sb = b.fp64only ? 0 : g.fixed ? S : choose_slices<S>(g.bst, task.block, b.kpad);
    asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(&g.cnt[4 + g.nblocks + task.block]), "r"(sb + 1)
                 : "memory");
  }
}
constexpr int kSliceThreads = 256;
template <int S, bool CPLX>
__global__ void __launch_bounds__(kSliceThreads, 2) gemm_split_slice_kernel(const FusedArgs args) {
  extern __shared__ __align__(16) unsigned char stage[];
  __shared__ int rexp[kStagedRowsMax];
  __shared__ unsigned long long wstat[2 * (kSliceThreads / 32)];
  const FusedArgs &g = args;
  pdl_wait();     // the operands come from earlier kernels of the stream
  pdl_trigger();  // the products launch may begin its prologue
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) TL_STAMP(28);
#pragma unroll 1
  for (int t = (int)blockIdx.x; t < g.nctasks; t += (int)gridDim.x) {
    const SliceTask task = g.stasks[t];
    slice_staged<S, CPLX, kSliceThreads>(task, task.operand == 0 ? (const void *)g.A : (const void *)g.B, g.ws,
                                         g.bst, stage, rexp, wstat);
    // publish the task's rows: the slices are read by bulk copies (async proxy) of the products
    fence_proxy_async_global();
    __syncthreads();
    if (threadIdx.x == 0) {
      publish_rows<S>(g, task);
      TL_ADD(30, 1);
    }
  }
  const int nw = (int)gridDim.x * (kSliceThreads / 32);
  for (int t = g.nctasks + (int)blockIdx.x * (kSliceThreads / 32) + (int)(threadIdx.x >> 5); t < g.nstasks; t += nw) {
    const SliceTask task = g.stasks[t];
    const void *X = task.operand == 0 ? (const void *)g.A : (const void *)g.B;
    [[maybe_unused]] const unsigned long long t0 = TL_NOW();
    slice_warp_task<S, CPLX>(task, X, g.ws, g.bst);
    fence_proxy_async_global();
    __syncwarp();
    if (lane == 0) {
      publish_rows<S>(g, task);
      TL_ADD(30, 1);
      TL_MAX(31, TL_NOW() - t0);
    }
  }
  // the slices are read by bulk copies (async proxy) of the products launch
  fence_proxy_async_global();
  if (lane == 0) TL_MAX(29, TL_NOW());
}

size_t tc_smem_bytes(int S) {
  return ring_stages(S) * (size_t)S * (PANEL_A + PANEL_B) * KSTAGE + kXchgBytes + kSmemTail;
}

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
  fa.hold0 = p->part_hold0;
  fa.err = ctx->counters + 8;
  fa.alpha = a;
  fa.beta = b;
  fa.nstasks = (int)p->nsrows;
  fa.nctasks = (int)p->nsctasks;
  fa.nitems = (int)p->nkstiles;
  fa.nblocks = (int)p->hblocks.size();
  fa.fixed = p->slices_fixed;
  const size_t smem = tc_smem_bytes(S);
  const bool bz = b.x == 0.0 && b.y == 0.0;
  auto k = cplx ? (bz ? gemm_split_fused_kernel<S, true, true> : gemm_split_fused_kernel<S, true, false>)
                : (bz ? gemm_split_fused_kernel<S, false, true> : gemm_split_fused_kernel<S, false, false>);
  TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (fa.nstasks > 0) {
    auto ks = cplx ? gemm_split_slice_kernel<S, true> : gemm_split_slice_kernel<S, false>;
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes));
    // one CTA per staged task and one warp per warp task, where that fits two CTAs per SM
    const int warps = kSliceThreads / 32;
    const int grid = std::max(1, std::min(2 * ctx->num_sms,
                                          std::max(fa.nctasks, (fa.nstasks - fa.nctasks + warps - 1) / warps)));
    TKB_CUDA_TRY(ctx, launch_pdl(ks, dim3((unsigned)grid), dim3(kSliceThreads), (size_t)kStageBytes, ctx->stream, fa));
    ctx->launches++;
  }
  // two-CTA clusters, as many as can be resident at once (the persistent loop takes the rest)
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ctx->num_sms & ~1));
  cfg.blockDim = dim3(kFusedThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  attr[1].id = cudaLaunchAttributeClusterDimension;
  attr[1].val.clusterDim.x = 2;
  attr[1].val.clusterDim.y = 1;
  attr[1].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> active;  // (kernel, device) → resident clusters
  int ncl = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair((const void *)k, ctx->device);
    auto f = active.find(key);
    if (f != active.end()) {
      ncl = f->second;
    } else {
      TKB_CUDA_TRY(ctx, cudaOccupancyMaxActiveClusters(&ncl, k, &cfg));
      active[key] = ncl;
    }
  }
  if (ncl < 1) return tkb_set_error(ctx, TKB_ERR_CUDA, "split GEMM: no two-CTA cluster fits an SM pair");
  cfg.gridDim = dim3((unsigned)(2 * std::min(ncl, ctx->num_sms / 2)));
  TKB_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, k, fa));
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

int64_t roundup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

}  // namespace

#ifdef TKB_TIMELINE
// copies the timeline of the last fused launch (kTlCtas × kTlSlots values) and clears it
extern "C" int tkb_timeline_read(unsigned long long *out) {
  if (cudaMemcpyFromSymbol(out, tkb_tl, sizeof(tkb_tl)) != cudaSuccess) return -1;
  static unsigned long long zero[kTlCtas * kTlSlots];
  return cudaMemcpyToSymbol(tkb_tl, zero, sizeof(tkb_tl)) == cudaSuccess ? kTlSlots : -1;
}
#endif

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
  // slicing tasks. Rows whose K values fit the stage go to staged CTA tasks of up to
  // kStagedRowsMax rows and kStageBytes of values, made smaller (down to one row) while there would
  // be fewer tasks than two per SM; longer rows go to warp tasks (about kTaskPieces pieces of whole
  // rows, in multiples of the rows one pass of the warp takes). CTA tasks come first; each list is
  // sorted largest first. Only the operands' own rows are sliced: padding rows of a panel feed
  // output rows and columns that are never stored.
  std::vector<SliceTask> jobs, wjobs;
  {
    const int64_t esize = cplx ? 16 : 8;
    int64_t staged_bytes = 0;
    for (const SJob &t : sj) {
      const int64_t kfull = cplx ? p->hblocks[t.block].kpad / 2 : p->hblocks[t.block].kpad;
      const int64_t rowb = (kfull + kfull / (cplx ? 8 : 16)) * esize;
      if (rowb <= kStageBytes) staged_bytes += rowb * t.nsrc;
    }
    const int64_t per_task = std::max<int64_t>(8 * 1024, staged_bytes / std::max<int64_t>(1, 2 * ctx->num_sms));
    for (const SJob &t : sj) {
      const int64_t kfull = cplx ? p->hblocks[t.block].kpad / 2 : p->hblocks[t.block].kpad;
      const int64_t rowb = (kfull + kfull / (cplx ? 8 : 16)) * esize;
      if (rowb <= kStageBytes) {
        const int32_t r = (int32_t)std::max<int64_t>(
            1, std::min<int64_t>({(int64_t)kStagedRowsMax, kStageBytes / rowb, (per_task + rowb - 1) / rowb}));
        for (int32_t r0 = 0; r0 < t.nsrc; r0 += r) {
          SliceTask j{};
          j.block = t.block;
          j.operand = t.op;
          j.r0 = r0;
          j.nrows = std::min(r, t.nsrc - r0);
          jobs.push_back(j);
        }
      } else {
        const int64_t R = 32 / slice_groups(t.nchunk);
        const int64_t passes = std::max<int64_t>(1, kTaskPieces / (R * std::max<int32_t>(1, t.nchunk)));
        const int32_t r = (int32_t)(R * passes);
        for (int32_t r0 = 0; r0 < t.nsrc; r0 += r) {
          SliceTask j{};
          j.block = t.block;
          j.operand = t.op;
          j.r0 = r0;
          j.nrows = std::min(r, t.nsrc - r0);
          wjobs.push_back(j);
        }
      }
    }
    auto cost = [&](const SliceTask &x) { return (int64_t)x.nrows * p->hblocks[x.block].kpad; };
    auto larger = [&](const SliceTask &x, const SliceTask &y) { return cost(x) > cost(y); };
    std::stable_sort(jobs.begin(), jobs.end(), larger);
    std::stable_sort(wjobs.begin(), wjobs.end(), larger);
    p->nsctasks = (int64_t)jobs.size();
    jobs.insert(jobs.end(), wjobs.begin(), wjobs.end());
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
  // the block fields every slicing task needs, in its own record
  for (SliceTask &j : jobs) {
    const GBlock &b = p->hblocks[j.block];
    const int opx = j.operand == 0 ? b.opA : b.opB;
    if (j.operand == 0) {
      j.xoff = b.offA;
      j.rs = opx == TKB_OP_N ? 1 : b.lda;
      j.ks = opx == TKB_OP_N ? b.lda : 1;
      j.ws_s = b.wsA;
      j.ws_e = b.wsEA;
      j.msrc = (int32_t)b.m;
    } else {
      j.xoff = b.offB;
      j.rs = opx == TKB_OP_N ? b.ldb : 1;
      j.ks = opx == TKB_OP_N ? 1 : b.ldb;
      j.ws_s = b.wsB;
      j.ws_e = b.wsEB;
      j.msrc = (int32_t)b.n;
    }
    j.k = (int32_t)b.k;
    j.kpad = b.kpad;
    j.conj = opx == TKB_OP_C ? 1 : 0;
  }
  off = roundup((int64_t)off, 256);
  std::stable_sort(tiles.begin(), tiles.end(), [&](const GTile &x, const GTile &y) {
    return p->hblocks[x.block].kpad > p->hblocks[y.block].kpad;
  });
  // products items in pairs, one pair per two-CTA cluster of the persistent kernel: a split tile
  // (its two K halves, one per CTA) or two unsplit tiles (the second may be empty). As many of the
  // longest tiles are split as keep the pairs within one cluster round (num_sms / 2 pairs), when
  // the decomposition allows it (max_pieces ≥ 2, halves of at least min_piece_steps stages). A tile
  // whose K needs more than one exact piece (int32 accumulators stay exact over (2^31 − 1)/(S·127²)
  // K positions) is split in any case; a block whose K needs more than two runs in FP64.
  std::vector<SplitTile> kt;
  int nslots = 0, npart = 0;
  {
    const int64_t maxst = std::max<int64_t>(1, (int64_t)2147483647 / ((int64_t)S * 127 * 127) / KSTAGE);
    const int64_t ncl = std::max<int64_t>(1, ctx->num_sms / 2);
    for (GBlock &b : p->hblocks)
      if (b.kpad / KSTAGE > 2 * maxst) b.fp64only = 1;
    const int64_t nt = (int64_t)tiles.size();
    int64_t budget = p->max_pieces >= 2 ? std::max<int64_t>(0, 2 * ncl - nt) : 0;  // tiles to split
    struct Pair {
      SplitTile a, b;
      int64_t cost;
    };
    std::vector<Pair> pairs;
    std::vector<SplitTile> singles;
    const SplitTile none{0, 0, 0, 2, 0, 0, -1, 1, 0, 0};
    for (const GTile &t : tiles) {  // longest K first
      const int nk = t.kind == 0 ? p->hblocks[t.block].kpad / KSTAGE : 0;
      const bool must = t.kind == 0 && nk > maxst && !p->hblocks[t.block].fp64only;
      const bool may = t.kind == 0 && budget > 0 && nk >= 2 * p->min_piece_steps;
      if (must || may) {
        if (!must) --budget;
        pairs.push_back({{t.block, t.m0, t.n0, 0, 0, nk / 2, -1, 2, 0, 0},
                         {t.block, t.m0, t.n0, 0, nk / 2, nk, -1, 2, 1, 0}, (int64_t)(nk - nk / 2)});
      } else {
        singles.push_back({t.block, t.m0, t.n0, t.kind, 0, nk, -1, 1, 0, 0});
      }
    }
    std::stable_sort(singles.begin(), singles.end(),
                     [](const SplitTile &x, const SplitTile &y) { return (x.ke - x.kb) > (y.ke - y.kb); });
    for (size_t q = 0; q < singles.size(); q += 2)
      pairs.push_back({singles[q], q + 1 < singles.size() ? singles[q + 1] : none, (int64_t)(singles[q].ke - singles[q].kb)});
    std::stable_sort(pairs.begin(), pairs.end(), [](const Pair &x, const Pair &y) { return x.cost > y.cost; });
    for (const Pair &pr : pairs) {
      kt.push_back(pr.a);
      kt.push_back(pr.b);
    }
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
  // one hold tile per CTA (β ≠ 0, one piece: the recombined values wait there for the tile check)
  p->part_hold0 = npart;
  if (e == cudaSuccess && !kt.empty())
    e = cudaMalloc((void **)&p->part, (size_t)(npart + ctx->num_sms) * 64 * 128 * sizeof(double));
  // claim, finish, check and slicing-warp counts, then one split-K arrival counter per split
  // tile; the block statistics; the per-block slice counts of the last launch
  const size_t nb = p->hblocks.size();
  const size_t ncnt = 4 + 2 * nb + (size_t)nslots;
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
