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
// Launches: slicing pass (32 source rows per task, run by 1–4 CTAs of a thread-block cluster:
// row maxima, exponents, slices) + product pass:
//   tcgen05 kernel (default): one CTA per 128×64 output tile (and K range, when the K loop
//   is split across CTAs); one thread streams the stages of A and B with cp.async.bulk into a
//   shared-memory ring as deep as fits (5 stages at S = 7) and issues tcgen05.mma.kind::i8
//   (M=128, K=32, N = 64 per B slice, up to four B slices per instruction) into S int32
//   diagonal accumulators held in tensor memory (S·64 of 512 columns); eight warps (two per
//   TMEM lane quarter) read the accumulators back with tcgen05.ld and recombine them in FP64.
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
constexpr int kSmemMax = 232448;             // dynamic shared memory per CTA (227 KiB)
// depth of the shared-memory ring: as many stages of S slices of A and B as fit, at most 8
__host__ __device__ constexpr int ring_stages(int S) {
  return (kSmemMax - 1024) / (S * (PANEL_A + PANEL_B) * KSTAGE) < 8
             ? (kSmemMax - 1024) / (S * (PANEL_A + PANEL_B) * KSTAGE)
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

// Slicing pass: one task = 32 source rows of one operand of one block over the whole K range,
// run by g of the kSliceCluster CTAs of a thread-block cluster (g sized so that every warp has
// about one warp tile, tasks packed into clusters by the host), which split the K range (the
// partial row maxima are combined through distributed shared memory). Source rows are the rows of op(A)
// and the columns of op(B) (for ComplexF64 a complex source row of op(A) gives the real row
// pair 2r, 2r+1). The cluster first reduces the row maxima (phase 1), derives the row
// exponents, then re-reads the rows (now cached) and writes the S slices (phase 2) as 8-byte
// pieces (8 consecutive K of one row) of the tensor-core operand layout.
//
// Every warp works on warp tiles; after loading, each lane holds LK consecutive K values of
// one source row, LK = 8 (small tiles: many warps per task and short per-warp chains, for
// slicing passes that fit one wave) or 16 (fewer instructions per value, for larger ones):
//   rows contiguous in memory (real op(A) = A, op(B) = Bᵀ; complex likewise): lane = row,
//     tile = 32 rows × LK K, loads straight from global memory (coalesced along rows);
//   K contiguous (op(A) = Aᵀ/Aᴴ, op(B) = B): lanes along K (coalesced), staged through a
//     per-warp shared-memory tile (one padding element per LK) and read back row-wise:
//     real 4 rows × 8·LK K, complex 8 rows × 4·LK K.
// ComplexF64 K is laid out as [Re | Im] halves of kh = round_up(k, 16) positions each, so an
// LK piece of the source maps to one piece in each half.
struct SliceTask {  // one entry per CTA
  int32_t block;
  int32_t operand;  // 0 = rows of op(A), 1 = columns of op(B), -1 = idle CTA
  int32_t r0;       // first source row
  int32_t sub;      // index of this CTA among the task's CTAs
  int32_t g;        // number of CTAs of the task
  int32_t rank0;    // cluster rank of the task's first CTA
};

constexpr int kSliceThreads = 256;
constexpr int kSliceCluster = 4;  // CTAs per thread-block cluster of the slicing pass
// bytes of one warp's staging tile (complex: 8 rows × 4·LK K of 16-byte values, one padding
// value per LK; real: half)
__host__ __device__ constexpr int slice_warp_smem(int LK) { return 8 * 4 * (LK + 1) * 16; }
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

// Warp tile t in two steps: fetch_tile issues the global loads into f[LK] (rows contiguous:
// the lane's row, K-contiguous: RG rows × NH values along K per lane, lanes along K), and
// unpack_tile turns them into v[LK] = LK consecutive K values of one source row, staging the
// K-contiguous layout through the warp's shared-memory tile. unpack returns the lane's source
// row (relative to the task) and the source K of v[0] through row/c, and false when the lane's
// piece lies beyond the padded K. Splitting the two lets a warp fetch its next tile while it
// slices the current one.
template <bool CPLX, bool ROWC, int LK>
__device__ __forceinline__ void fetch_tile(int t, const typename SrcVal<CPLX>::T *__restrict__ X, int64_t xo,
                                           int64_t rs, int64_t ks, int64_t r0, int64_t msrc, int64_t ksrc,
                                           int lane, typename SrcVal<CPLX>::T (&f)[LK]) {
  using T = typename SrcVal<CPLX>::T;
  const T z = zero_of(T{});
  if constexpr (ROWC) {
    const int64_t c = LK * (int64_t)t;
    const int64_t r = r0 + lane;
    const bool rv = r < msrc;
    const T *p = X + xo + r * rs;
#pragma unroll
    for (int q = 0; q < LK; ++q) f[q] = (rv && c + q < ksrc) ? __ldg(p + (c + q) * ks) : z;
  } else {
    constexpr int RG = CPLX ? 8 : 4;         // rows per warp tile
    constexpr int KW = (CPLX ? 4 : 8) * LK;  // K per warp tile
    constexpr int NH = KW / 32;              // loads per row per lane
    static_assert(RG * NH == LK, "one fetched value per unpacked value");
    const int ngrp = 32 / RG;
    const int grp = t % ngrp;
    const int64_t k0 = (int64_t)(t / ngrp) * KW;
#pragma unroll
    for (int rr = 0; rr < RG; ++rr) {
      const int64_t r = r0 + grp * RG + rr;
      const bool rv = r < msrc;
      const T *p = X + xo + r * rs;
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const int64_t l = k0 + 32 * h + lane;
        f[rr * NH + h] = (rv && l < ksrc) ? __ldg(p + l) : z;
      }
    }
  }
}
template <bool CPLX, bool ROWC, int LK>
__device__ __forceinline__ bool unpack_tile(int t, const typename SrcVal<CPLX>::T (&f)[LK], int64_t kfull,
                                            typename SrcVal<CPLX>::T *stage, int lane,
                                            typename SrcVal<CPLX>::T (&v)[LK], int &row, int64_t &c) {
  if constexpr (ROWC) {
#pragma unroll
    for (int q = 0; q < LK; ++q) v[q] = f[q];
    row = lane;
    c = LK * (int64_t)t;
    return true;
  } else {
    constexpr int RG = CPLX ? 8 : 4;
    constexpr int KW = (CPLX ? 4 : 8) * LK;
    constexpr int NH = KW / 32;
    constexpr int RP = (KW / LK) * (LK + 1);  // staging row pitch (elements)
    const int ngrp = 32 / RG;
    const int grp = t % ngrp;
    const int64_t k0 = (int64_t)(t / ngrp) * KW;
    __syncwarp();
#pragma unroll
    for (int rr = 0; rr < RG; ++rr)
#pragma unroll
      for (int h = 0; h < NH; ++h)
        stage[rr * RP + ((32 / LK) * h + lane / LK) * (LK + 1) + lane % LK] = f[rr * NH + h];
    __syncwarp();
    constexpr int LPR = 32 / RG;  // lanes per row
    static_assert(LPR * LK == KW, "one warp tile row is read back by LPR lanes");
    const int rr = lane / LPR, kap = lane % LPR;
#pragma unroll
    for (int q = 0; q < LK; ++q) v[q] = stage[rr * RP + kap * (LK + 1) + q];
    row = grp * RG + rr;
    c = k0 + LK * kap;
    return c < kfull;
  }
}
template <bool CPLX, bool ROWC, int LK>
__device__ __forceinline__ bool load_tile(int t, const typename SrcVal<CPLX>::T *__restrict__ X,
                                          int64_t xo, int64_t rs, int64_t ks, int64_t r0,
                                          int64_t msrc, int64_t ksrc, int64_t kfull,
                                          typename SrcVal<CPLX>::T *stage, int lane,
                                          typename SrcVal<CPLX>::T (&v)[LK], int &row, int64_t &c) {
  typename SrcVal<CPLX>::T f[LK];
  fetch_tile<CPLX, ROWC, LK>(t, X, xo, rs, ks, r0, msrc, ksrc, lane, f);
  return unpack_tile<CPLX, ROWC, LK>(t, f, kfull, stage, lane, v, row, c);
}

// Phase-1 row maxima of warp tile t of a K-contiguous source (the layout load_tile stages):
// each lane reduces its own values per row, then the warp takes the maximum per row with two
// 32-bit max-reductions (high word, then low word among the lanes holding the high maximum;
// the bits of non-negative doubles order like their values). No staging, so the loads of
// consecutive tiles can overlap.
template <bool CPLX, int LK>
__device__ __forceinline__ void tile_rowmax_kc(int t, const typename SrcVal<CPLX>::T *__restrict__ X, int64_t xo,
                                               int64_t rs, int64_t r0, int64_t msrc, int64_t ksrc, int lane,
                                               unsigned long long *rmax) {
  using T = typename SrcVal<CPLX>::T;
  const T z = zero_of(T{});
  constexpr int RG = CPLX ? 8 : 4;
  constexpr int KW = (CPLX ? 4 : 8) * LK;
  constexpr int NH = KW / 32;
  const int ngrp = 32 / RG;
  const int grp = t % ngrp;
  const int64_t k0 = (int64_t)(t / ngrp) * KW;
  double m[RG];
#pragma unroll
  for (int rr = 0; rr < RG; ++rr) {
    const int64_t r = r0 + grp * RG + rr;
    const bool rv = r < msrc;
    const T *p = X + xo + r * rs;
    double mm = 0.0;
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      const int64_t l = k0 + 32 * h + lane;
      mm = fmax(mm, absmax((rv && l < ksrc) ? __ldg(p + l) : z));
    }
    m[rr] = mm;
  }
#pragma unroll
  for (int rr = 0; rr < RG; ++rr) {
    const unsigned hi = (unsigned)__double2hiint(m[rr]), lo = (unsigned)__double2loint(m[rr]);
    const unsigned H = __reduce_max_sync(0xffffffffu, hi);
    const unsigned L = __reduce_max_sync(0xffffffffu, hi == H ? lo : 0u);
    if (lane == rr && (H | L) != 0u)
      atomicMax(&rmax[grp * RG + rr], ((unsigned long long)H << 32) | (unsigned long long)L);
  }
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

// thread-block cluster helpers (the K range of a task is split over the CTAs of a cluster)
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// 64-bit load from the shared memory of CTA `rank` of this cluster, at the address that `p`
// has in this CTA
__device__ __forceinline__ unsigned long long ld_dsmem_u64(const void *p, uint32_t rank) {
  uint32_t remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n"
               : "=r"(remote)
               : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
  unsigned long long v;
  asm volatile("ld.shared::cluster.u64 %0, [%1];\n" : "=l"(v) : "r"(remote) : "memory");
  return v;
}

template <int S, bool CPLX, bool ROWC, int LK>
__device__ __forceinline__ void slice_task(const GBlock &b, const SliceTask &task, const void *Xv, int8_t *ws,
                                           unsigned char *wsmem, unsigned long long *rmax, int *rexp) {
  using T = typename SrcVal<CPLX>::T;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int op = task.operand;
  const int64_t r0 = task.r0;
  // the task's CTAs share its warp tiles: sub·8 + warp, then every 8·g
  const uint32_t crank = cluster_rank();
  const int t0 = task.sub * (kSliceThreads / 32) + warp;
  const int tstep = task.g * (kSliceThreads / 32);
  const T *X = reinterpret_cast<const T *>(Xv);
  T *stage = reinterpret_cast<T *>(wsmem + warp * (CPLX ? slice_warp_smem(LK) : slice_warp_smem(LK) / 2));
  const int64_t xo = op == 0 ? b.offA : b.offB;
  const int opx = op == 0 ? b.opA : b.opB;
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
  const int ntile = ROWC ? (int)(kfull / LK)
                         : (CPLX ? 4 : 8) * (int)((kfull + (CPLX ? 4 : 8) * LK - 1) / ((CPLX ? 4 : 8) * LK));

  // phase 1: row maxima of this CTA's tiles. With 8-K real tiles the warp's first tile stays
  // in registers for phase 2 (most warps have one tile).
  constexpr bool KEEP = LK == 8 && !CPLX && ROWC;
  T keep[KEEP ? LK : 1];
#pragma unroll 2
  for (int t = t0; t < ntile; t += tstep) {
    if constexpr (!ROWC) {
      tile_rowmax_kc<CPLX, LK>(t, X, xo, rs, r0, msrc, b.k, lane, rmax);
      continue;
    }
    T v[LK];
    int row;
    int64_t c;
    const bool ok = load_tile<CPLX, ROWC, LK>(t, X, xo, rs, ks, r0, msrc, b.k, kfull, stage, lane, v, row, c);
    if constexpr (KEEP) {
      if (t == t0) {
#pragma unroll
        for (int q = 0; q < LK; ++q) keep[q] = v[q];
      }
    }
    double m = 0.0;
#pragma unroll
    for (int q = 0; q < LK; ++q) m = fmax(m, absmax(v[q]));
    if (m > 0.0) atomicMax(&rmax[row], (unsigned long long)__double_as_longlong(m));
  }
  // partial maxima of the task's CTAs → row exponents (written by the task's first CTA)
  __syncthreads();
  cluster_arrive();
  cluster_wait();
  if (tid < 32) {
    unsigned long long mb = rmax[tid];
    for (uint32_t q = (uint32_t)task.rank0; q < (uint32_t)(task.rank0 + task.g); ++q)
      if (q != crank) mb = max(mb, ld_dsmem_u64(&rmax[tid], q));
    const int e = row_exponent<S>(__longlong_as_double((long long)mb));
    rexp[tid] = e;
    int32_t *ex = reinterpret_cast<int32_t *>(ws + (op == 0 ? b.wsEA : b.wsEB));
    const int64_t r = r0 + tid;
    if (task.sub == 0) {
      if (CPLX && op == 0) {
        ex[2 * r] = e;
        ex[2 * r + 1] = e;
      } else {
        ex[r] = e;
      }
    }
  }
  // done reading the peers' maxima (no ordering needed: relaxed); the matching wait before exit
  // keeps every CTA's shared memory alive until all peers have read it
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
  __syncthreads();

  // phase 2: slices
  const int pr = op == 0 ? PANEL_A : PANEL_B;
  const int64_t kpad = b.kpad;
  int8_t *base = ws + (op == 0 ? b.wsA : b.wsB);
  const int64_t plane = (int64_t)pr * KSTAGE;  // between the slices of one stage
  // the next tile is fetched before the current one is sliced (its loads overlap the work)
  T nxt[LK];
  if (t0 < ntile) {
    if (KEEP) {
#pragma unroll
      for (int q = 0; q < LK; ++q) nxt[q] = keep[KEEP ? q : 0];
    } else {
      fetch_tile<CPLX, ROWC, LK>(t0, X, xo, rs, ks, r0, msrc, b.k, lane, nxt);
    }
  }
  for (int t = t0; t < ntile; t += tstep) {
    T cur[LK];
#pragma unroll
    for (int q = 0; q < LK; ++q) cur[q] = nxt[q];
    if (t + tstep < ntile) fetch_tile<CPLX, ROWC, LK>(t + tstep, X, xo, rs, ks, r0, msrc, b.k, lane, nxt);
    T v[LK];
    int row;
    int64_t c;
    const bool ok = unpack_tile<CPLX, ROWC, LK>(t, cur, kfull, stage, lane, v, row, c);
    if (!ok) continue;
    const RowScale rsc = row_scale<S>(rexp[row]);
    const int64_t r = r0 + row;
    // one slice per iteration (not unrolled: the body is reused S times, which keeps the
    // code of this short-lived kernel small)
    if constexpr (!CPLX) {
      using P = typename Piece<LK>::T;
      Fixed x[LK];
      uint32_t M[LK / 4];
#pragma unroll
      for (int q = 0; q < LK; ++q) x[q] = to_fixed(v[q], rsc);
      sign_masks([&](int q) { return v[q]; }, M);
      int8_t *p = base + slice_off(r, c, kpad, pr, S);
#pragma unroll 1
      for (int sl = 0; sl < S; ++sl, p += plane) *reinterpret_cast<P *>(p) = slice_piece<S, LK>(x, M, sl);
    } else {
      using P = typename Piece<LK>::T;
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
#pragma unroll 1
        for (int sl = 0; sl < S; ++sl) {
          const P ur = slice_piece<S, LK>(xr, Mr, sl);
          const int64_t o = sl * plane;
          *reinterpret_cast<P *>(p0 + o) = ur;
          *reinterpret_cast<P *>(p1 + o) = slice_piece<S, LK>(xi, Mn, sl);
          *reinterpret_cast<P *>(p2 + o) = slice_piece<S, LK>(xi, Mi, sl);
          *reinterpret_cast<P *>(p3 + o) = ur;
        }
      } else {        // column j of op(B): [Re | Im]
        int8_t *p0 = base + slice_off(r, c, kpad, pr, S);
        int8_t *p1 = base + slice_off(r, kfull + c, kpad, pr, S);
#pragma unroll 1
        for (int sl = 0; sl < S; ++sl) {
          const int64_t o = sl * plane;
          *reinterpret_cast<P *>(p0 + o) = slice_piece<S, LK>(xr, Mr, sl);
          *reinterpret_cast<P *>(p1 + o) = slice_piece<S, LK>(xi, Mi, sl);
        }
      }
    }
  }
  cluster_wait();
}

template <int S, bool CPLX, int LK>
__global__ void __launch_bounds__(kSliceThreads, LK == 8 ? (CPLX ? 2 : 3) : (CPLX ? 1 : 2))
    slice_kernel(const GBlock *__restrict__ blocks, const SliceTask *__restrict__ tasks,
                 const double *__restrict__ A, const double *__restrict__ B, int8_t *ws) {
  extern __shared__ __align__(16) unsigned char slice_smem[];
  __shared__ unsigned long long rmax[32];
  __shared__ int rexp[32];
  pdl_wait();     // the operands come from the previous kernel of the stream
  pdl_trigger();  // the product kernel may be scheduled (it waits for this grid to finish)
  const SliceTask task = tasks[blockIdx.x];
  const int op = task.operand;
  if (op < 0) {  // idle CTA: the cluster barriers of the task CTAs (two phases) still count it
    cluster_arrive();
    cluster_wait();
    cluster_arrive();
    cluster_wait();
    return;
  }
  const GBlock &b = blocks[task.block];
  if (threadIdx.x < 32) rmax[threadIdx.x] = 0ull;
  __syncthreads();
  const int opx = op == 0 ? b.opA : b.opB;
  const bool rowc = op == 0 ? opx == TKB_OP_N : opx != TKB_OP_N;
  const void *X = op == 0 ? (const void *)A : (const void *)B;
  if (rowc) slice_task<S, CPLX, true, LK>(b, task, X, ws, slice_smem, rmax, rexp);
  else slice_task<S, CPLX, false, LK>(b, task, X, ws, slice_smem, rmax, rexp);
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
// bounded wait until *p ≥ target (acquire at GPU scope); false once 2 s have passed
__device__ __forceinline__ bool wait_count(const int *p, int target) {
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    if (v >= target) return true;
    if (globaltimer_ns() - t0 > 2000000000ull) return false;
    __nanosleep(32);
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
// tcgen05.ld without the wait; tmem_ld_wait on the same registers orders their uses after it
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                 "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                 "+r"(r[14]), "+r"(r[15])
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

// One product task: output tile (m0, n0) of a block, K stages [kb, ke). When a tile's K
// range is split over nsplit CTAs (few tiles, long K), each CTA recombines its own int32
// diagonals into an FP64 partial tile, and the partials are added in split order
// (deterministic) before the scaling and the store to C:
//   CL = true: the pieces of a tile are the CTAs of one thread-block cluster; each keeps its
//     partial in its own (now idle) ring memory, and after a cluster barrier CTA `sid` reduces
//     the column chunks sid, sid + nsplit, … of the tile through distributed shared memory.
//     Clusters without a split tile hold up to cluster-size independent tiles (or idle CTAs,
//     kind 2).
//   CL = false: each piece stores its partial (plain coalesced stores) in partial buffer
//     pbase + sid; when the launch is one wave, every piece waits for the others and reduces a
//     share of the column chunks, otherwise the CTA that arrives last on the tile's counter
//     adds all partials (any number of pieces).
struct SplitTile {
  int32_t block, m0, n0, kind;
  int32_t kb, ke, slot, nsplit;
  int32_t sid, pbase;
};

__device__ __forceinline__ uint32_t mapa_u32(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ double ld_dsmem_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];\n" : "=d"(v) : "r"(addr) : "memory");
  return v;
}

constexpr int kTcThreads = 256;

template <int S, bool CL>
__global__ void __launch_bounds__(kTcThreads, 1)
    gemm_split_tc_kernel(const GBlock *__restrict__ blocks, const SplitTile *__restrict__ tiles,
                         const int8_t *__restrict__ ws, int cplx, double *__restrict__ C, CDbl alpha,
                         CDbl beta, int *err, double *__restrict__ part, int *__restrict__ pcnt, int spin) {
  constexpr uint32_t A_BYTES = S * PANEL_A * KSTAGE, B_BYTES = S * PANEL_B * KSTAGE;
  constexpr uint32_t STAGE = A_BYTES + B_BYTES;
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr int NSTAGE = ring_stages(S);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * STAGE);
  uint64_t *empty = full + NSTAGE;
  uint64_t *done = full + 2 * NSTAGE;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(full + 2 * NSTAGE + 1);
  int *ticket = reinterpret_cast<int *>(full + 2 * NSTAGE + 2);
  int *ebs = reinterpret_cast<int *>(full + 2 * NSTAGE + 4);  // column exponents of the tile
  double *cscale = reinterpret_cast<double *>(full + 2 * NSTAGE + 36);  // 2^(column exponent)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const SplitTile tile = tiles[blockIdx.x];
  const GBlock b = blocks[tile.block];
  const bool has_k = tile.kind == 0;
  const bool idle = CL && tile.kind == 2;  // padding CTA of a cluster
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
  pdl_wait();  // slices and exponents come from the slicing kernel (set-up above overlapped it)
  if (tid >= 64 && tid < 128) {  // column exponents into shared memory while warp 0 starts the products
    const int col = tid - 64;
    const int64_t j = tile.n0 + col;
    const int ej = (has_k && j < b.n) ? max(reinterpret_cast<const int32_t *>(ws + b.wsEB)[j], -1100) : 0;
    ebs[col] = ej;
    cscale[col] = (ej >= -1022 && ej <= 1023) ? pow2i(ej) : 0.0;  // 0: scale through ldexp
  }

  // producer: lane 0 of warp 0; the other lanes of warp 0 wait at the __syncwarp below (no
  // polling that would take issue slots from the producer)
  if (has_k && tid == 0) {
    const int8_t *gA = ws + b.wsA + (int64_t)(tile.m0 / PANEL_A) * S * PANEL_A * b.kpad;
    const int8_t *gB = ws + b.wsB + (int64_t)(tile.n0 / PANEL_B) * S * PANEL_B * b.kpad;
    auto load = [&](int kt, int st) {  // kt: local stage index, global stage kb + kt
      unsigned char *sa = smem + st * STAGE;
      const int64_t kg = kb + kt;
      mbar_expect_tx(&full[st], STAGE);
      bulk_g2s(sa, gA + kg * A_BYTES, A_BYTES, &full[st]);
      bulk_g2s(sa + A_BYTES, gB + kg * B_BYTES, B_BYTES, &full[st]);
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
        for (int t = 0; t < S - s; t += kMaxSlicesPerMma) {
          const int nsl = (S - s - t) < kMaxSlicesPerMma ? (S - s - t) : kMaxSlicesPerMma;
          umma_i8(tmem + (uint32_t)((s + t) * 64), ad[s], bd[t], idesc_i8(64u * (uint32_t)nsl),
                  (kt > 0 || s > 0) ? 1u : 0u);
        }
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
  if (warp == 0) __syncwarp();
  if (has_k) {
    if (!mbar_wait(done, 0)) atomicExch(err, 2);
    tc_fence_after();
  }
  __syncwarp();  // tcgen05.ld is warp-collective: reconverge after the divergent waits
  __syncthreads();  // ebs visible; every warp is past its wait
  // epilogue: warp w owns accumulator rows 32(w mod 4) .. 32(w mod 4) + 31 (the TMEM lanes its
  // warp may read) and the column chunks 2·half, 2·half + 1 (16 columns each), half = w / 4
  const int32_t *eA = reinterpret_cast<const int32_t *>(ws + b.wsEA);
  const int64_t Mreal = cplx ? 2 * b.m : b.m;
  const int row = 32 * (warp & 3) + lane;
  const int half = warp >> 2;
  const int64_t i = tile.m0 + row;
  const int ei = (has_k && i < Mreal) ? max(eA[i], -1100) : 0;
  const double rscale = (ei >= -1022 && ei <= 1023) ? pow2i(ei) : 0.0;
  // this CTA's FP64 recombination of its diagonals: chunk c of 16 columns
  auto recombine = [&](int c, double (&v)[16]) {
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = 0.0;
    if (!has_k) return;
    // all S loads in flight, then one wait (the first wait covers every load issued before it)
    uint32_t r[S][16];
#pragma unroll
    for (int d = 0; d < S; ++d)
      tmem_ld16_issue(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(d * 64 + c * 16), r[d]);
#pragma unroll
    for (int d = 0; d < S; ++d) tmem_ld_wait(r[d]);
    // exact integer recombination: diagonals d = 0..2, 3..4, 5..6 are combined by Horner's
    // rule in base 128 into three int64 groups (each below 2^46 in magnitude), each turned
    // into a double without a conversion instruction, then scaled and summed in FP64
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      int64_t g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
      for (int d = 0; d < S; ++d) {
        const int64_t pd = (int32_t)r[d][q];
        if (d < 3) g0 = g0 * 128 + pd;
        else if (d < 5) g1 = g1 * 128 + pd;
        else g2 = g2 * 128 + pd;
      }
      double acc = i2d_small(g0) * pow2i(-7 * ((S < 3 ? S : 3) + 1));
      if (S > 3) acc = fma(i2d_small(g1), pow2i(-7 * ((S < 5 ? S : 5) + 1)), acc);
      if (S > 5) acc = fma(i2d_small(g2), pow2i(-7 * (S + 1)), acc);
      v[q] = acc;
    }
  };
  // Every row exponent and column exponent of the tile in the normal range (the common case):
  // the final scaling is two exact multiplications by powers of two; otherwise ldexp.
  int any_slow = (has_k && rscale == 0.0) ? 1 : 0;
  if (has_k && lane < 16 && warp == 0)
    any_slow |= (cscale[4 * lane] == 0.0 || cscale[4 * lane + 1] == 0.0 || cscale[4 * lane + 2] == 0.0 ||
                 cscale[4 * lane + 3] == 0.0) ? 1 : 0;
  const bool slow = __syncthreads_or(any_slow) != 0;
  // final values of chunk c: exponent scaling, α/β update, store to C (real: every old
  // value of C is loaded before the first store, so no load waits behind a store)
  auto final_store = [&](int c, double (&v)[16]) {
    if (has_k) {
      if (!slow) {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = v[q] * rscale * cscale[c * 16 + q];
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = scale2(v[q], ei + ebs[c * 16 + q]);
      }
    }
    if (!cplx) {
      const int64_t j0 = tile.n0 + c * 16;
      const int nj = (int)min((int64_t)16, b.n - j0);
      if (i >= b.m || nj <= 0) return;
      double *pc = C + b.offC + i + j0 * b.ldc;
      if (bz) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (q < nj) pc[q * b.ldc] = alpha.x * v[q];
      } else {
        double old[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) old[q] = q < nj ? pc[q * b.ldc] : 0.0;
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (q < nj) pc[q * b.ldc] = fma(beta.x, old[q], alpha.x * v[q]);
      }
      return;
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) store_out(v[q], i, tile.n0 + c * 16 + q, b, cplx, C, alpha, beta, bz, 1);
  };
  if constexpr (CL) {
    // the ring is idle (every stage landed and every product completed): it holds this CTA's
    // FP64 partial tile, [column][row]
    double *P = reinterpret_cast<double *>(smem);
    const bool split = tile.nsplit > 1;
    if (!idle) {
      if (split) asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
#pragma unroll 1
      for (int c = 2 * half; c < 2 * half + 2; ++c) {
        double v[16];
        recombine(c, v);
        if (split) {
#pragma unroll
          for (int q = 0; q < 16; ++q) P[(c * 16 + q) * 128 + row] = v[q];
        } else {
          final_store(c, v);
        }
      }
    }
    // a cluster holds either the pieces of one split tile or unsplit tiles only, so `split`
    // is uniform over the cluster: clusters of unsplit tiles skip both barriers
    if (split) {
      cluster_arrive();
      cluster_wait();
      const uint32_t pb = smem_u32(P) + (uint32_t)row * 8u;
#pragma unroll 1
      for (int c = tile.sid + half * tile.nsplit; c < 4; c += 2 * tile.nsplit) {
        double v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = 0.0;
#pragma unroll 1
        for (int sp = 0; sp < tile.nsplit; ++sp) {  // split order: deterministic sum
          const uint32_t rb = mapa_u32(pb, (uint32_t)sp) + (uint32_t)(c * 16 * 128 * 8);
          double t[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) t[q] = ld_dsmem_f64(rb + (uint32_t)(q * 128 * 8));
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] += t[q];
        }
        final_store(c, v);
      }
      // no CTA leaves while a peer may still read its partial
      cluster_arrive();
      cluster_wait();
    }
  } else {
  // Pass 0 (split tiles): recombine and store this CTA's FP64 partial tile. Pass 1 adds the
  // partials in split order (deterministic) and writes C:
  //   spin (the launch is one wave, one CTA per SM, so all pieces are resident): every piece
  //     waits (bounded) until all partials are stored, then takes its share of the column
  //     chunks (sid, sid + nsplit, …);
  //   otherwise the piece that arrives last on the tile's counter does all chunks.
  // Unsplit tiles run pass 1 on their own diagonals. One loop body, so each step is emitted
  // once.
  double *mine = part + (int64_t)(tile.pbase + tile.sid) * (64 * 128);  // [col][row]
  const bool split = tile.nsplit > 1;
  int pass = split ? 0 : 1;
  while (true) {
    const bool share = pass == 1 && split && spin;
    const int c0 = share ? tile.sid + half * tile.nsplit : 2 * half;
    const int cstep = share ? 2 * tile.nsplit : 1;
    const int cend = share ? 4 : 2 * half + 2;
#pragma unroll 1
    for (int c = c0; c < cend; c += cstep) {
      double v[16];
      if (pass == 0 || !split) {
        recombine(c, v);
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = 0.0;
#pragma unroll 4
        for (int sp = 0; sp < tile.nsplit; ++sp) {  // split order: deterministic sum
          const double *src = part + (int64_t)(tile.pbase + sp) * (64 * 128);
          double t[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) t[q] = __ldcg(&src[(c * 16 + q) * 128 + row]);
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] += t[q];
        }
      }
      if (pass == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) __stcg(&mine[(c * 16 + q) * 128 + row], v[q]);
      } else {
        final_store(c, v);
      }
    }
    if (pass == 1) break;
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      *ticket = atomicAdd(&pcnt[2 * tile.slot], 1);
      if (spin && !wait_count(&pcnt[2 * tile.slot], tile.nsplit)) atomicExch(err, 3);
    }
    __syncthreads();
    if (!spin && *ticket != tile.nsplit - 1) break;
    __threadfence();
    pass = 1;
  }
  // counters back to zero for the next launch: by the last piece through pass 1 (spin), or by
  // the piece that ran it
  if (split && tid == 0 && pass == 1) {
    if (!spin || atomicAdd(&pcnt[2 * tile.slot + 1], 1) == tile.nsplit - 1) {
      pcnt[2 * tile.slot] = 0;
      pcnt[2 * tile.slot + 1] = 0;
    }
  }
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
  for (int c = threadIdx.x; c < 2 * S * 128; c += blockDim.x) {
    const int op = c / (S * 128);
    const int rem = c % (S * 128);
    const int s = rem / 128, q = rem % 128;
    const int row = q >> 1, half = q & 1;
    if (op == 0) {
      const int8_t *g = ws + b.wsA + s * (PANEL_A * KSTAGE) + slice_off(m0 + row, k0 + half * 16, b.kpad, PANEL_A, S);
      cp_async16(As + (s * SBM + row) * SPITCH + half * 16, g);
    } else {
      const int8_t *g = ws + b.wsB + s * (PANEL_B * KSTAGE) + slice_off(n0 + row, k0 + half * 16, b.kpad, PANEL_B, S);
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
                for (int d = S - 1; d >= 0; --d)
                  v = fma((double)acc[d][mt][nt][hr * 2 + hc], pow2i(-7 * (d + 2)), v);
                v = scale2(v, ((i < Mreal) ? max(eA[i], -1100) : 0) + ((j < b.n) ? max(eB[j], -1100) : 0));
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

size_t tc_smem_bytes(int S) { return ring_stages(S) * (size_t)S * (PANEL_A + PANEL_B) * KSTAGE + 1024; }

bool use_mma_sync() {
  const char *e = std::getenv("TKB_SPLIT_KERNEL");
  return e && std::strcmp(e, "mma") == 0;
}

template <int S>
int launch_split(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B, CDbl a, CDbl b) {
  const int cplx = p->dtype == TKB_C128 ? 1 : 0;
  if (p->nsrows > 0) {
    // complex tiles stage 16-byte elements: twice the shared memory of real ones
    const int lk = p->slice_lk;
    const size_t smem = (size_t)(kSliceThreads / 32) * slice_warp_smem(lk) / (cplx ? 1 : 2);
    auto k = lk == 8 ? (cplx ? slice_kernel<S, true, 8> : slice_kernel<S, false, 8>)
                     : (cplx ? slice_kernel<S, true, 16> : slice_kernel<S, false, 16>);
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)p->nsrows);
    cfg.blockDim = dim3(kSliceThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kSliceCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    TKB_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, k, (const GBlock *)p->blocks, (const SliceTask *)p->sjobs,
                                         (const double *)A, (const double *)B, (int8_t *)ctx->ws));
    ctx->launches++;
    TKB_CUDA_TRY(ctx, cudaGetLastError());
  }
  if (use_mma_sync()) {
    for (const GBlock &hb : p->hblocks)
      if (!hb.skinny && (int64_t)hb.kpad * S * 127 * 127 > 2147483647ll)
        return tkb_set_error(ctx, TKB_ERR_UNSUPPORTED, "mma.sync split kernel: K too long for exact int32 products");
    const size_t smem = 2 * (size_t)(2 * S * SBM * SPITCH);
    auto k = gemm_split_mma_kernel<S>;
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (int)std::min<int64_t>(p->nstiles, (int64_t)ctx->num_sms * 2);
    k<<<grid, 256, smem, ctx->stream>>>(p->blocks, p->stiles, (int)p->nstiles, ctx->counters,
                                        (const int8_t *)ctx->ws, cplx, (double *)C, a, b);
  } else {
    const size_t smem = tc_smem_bytes(S);
    const bool cl = p->kcluster > 1;
    auto k = cl ? gemm_split_tc_kernel<S, true> : gemm_split_tc_kernel<S, false>;
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // programmatic dependent launch: barrier set-up and TMEM allocation overlap the slicing
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)p->nkstiles);
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[2];
    int na = 0;
    if (p->nsrows > 0) {
      attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[na++].val.programmaticStreamSerializationAllowed = 1;
    }
    if (cl) {
      attr[na].id = cudaLaunchAttributeClusterDimension;
      attr[na].val.clusterDim.x = (unsigned)p->kcluster;
      attr[na].val.clusterDim.y = 1;
      attr[na++].val.clusterDim.z = 1;
    }
    cfg.attrs = attr;
    cfg.numAttrs = na;
    TKB_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, k, (const GBlock *)p->blocks, (const SplitTile *)p->kstiles,
                                         (const int8_t *)ctx->ws, cplx, (double *)C, a, b, ctx->counters + 8,
                                         p->part, p->pcnt, p->kspin));
  }
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}

int64_t roundup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Co-resident clusters of the slicing pass (kSliceCluster CTAs each)
template <int S, bool CPLX, int LK>
int max_slice_clusters_t(cudaStream_t st) {
  auto k = slice_kernel<S, CPLX, LK>;
  const size_t smem = (size_t)(kSliceThreads / 32) * slice_warp_smem(LK) / (CPLX ? 1 : 2);
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)kSliceCluster);
  cfg.blockDim = dim3(kSliceThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kSliceCluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
template <int S>
int max_slice_clusters_s(bool cplx, int lk, cudaStream_t st) {
  if (lk == 8) return cplx ? max_slice_clusters_t<S, true, 8>(st) : max_slice_clusters_t<S, false, 8>(st);
  return cplx ? max_slice_clusters_t<S, true, 16>(st) : max_slice_clusters_t<S, false, 16>(st);
}
int max_slice_clusters(int S, bool cplx, int lk, cudaStream_t st, int num_sms) {
  int n = 0;
  switch (S) {
    case 3: n = max_slice_clusters_s<3>(cplx, lk, st); break;
    case 4: n = max_slice_clusters_s<4>(cplx, lk, st); break;
    case 5: n = max_slice_clusters_s<5>(cplx, lk, st); break;
    case 6: n = max_slice_clusters_s<6>(cplx, lk, st); break;
    default: n = max_slice_clusters_s<7>(cplx, lk, st); break;
  }
  return n > 0 ? n : num_sms / kSliceCluster;
}

// Co-resident thread-block clusters of `cs` product CTAs (one CTA per SM; clusters stay within
// one GPC, so this is below num_sms / cs on parts whose GPCs have SM counts not divisible by cs).
template <int S>
int max_clusters_t(int cs, cudaStream_t st) {
  auto k = gemm_split_tc_kernel<S, true>;
  const size_t smem = tc_smem_bytes(S);
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cs);
  cfg.blockDim = dim3(kTcThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
int max_clusters(int S, int cs, cudaStream_t st) {
  switch (S) {
    case 3: return max_clusters_t<3>(cs, st);
    case 4: return max_clusters_t<4>(cs, st);
    case 5: return max_clusters_t<5>(cs, st);
    case 6: return max_clusters_t<6>(cs, st);
    default: return max_clusters_t<7>(cs, st);
  }
}

// Cluster split plan: tiles with more than T stages are cut into cs pieces (one cluster each),
// the others are grouped cs per cluster in order of decreasing K (padded with idle CTAs).
// Cost model (tenths of a microsecond, from the measured epilogues): a K stage 10 (measured
// 0.7–1.1 us depending on the MMA grouping; the choices below did not change between the two),
// the epilogue of an unsplit tile 30, of a cluster-reduced piece 48, of a global-memory-reduced
// piece 57 + 3 per piece beyond two.
constexpr int64_t kCostStage = 10, kCostEpi = 30, kCostEpiCluster = 48, kCostEpiGlobal = 57, kCostEpiGlobalPiece = 3;
struct ClusterPlan {
  int cs = 0;
  int64_t T = 0, cost = INT64_MAX, ctas = 0;
};
ClusterPlan plan_clusters(const std::vector<int64_t> &nks, int S, int64_t maxst, int64_t nsm, cudaStream_t st) {
  ClusterPlan best;
  const int64_t nt = (int64_t)nks.size();  // stages per tile, decreasing (0: no products)
  for (int cs = 2; cs <= 4; ++cs) {
    const int64_t cap = std::min<int64_t>(max_clusters(S, cs, st), nsm / cs);
    if (cap <= 0) continue;
    // candidate thresholds: split the first ns tiles (those with the most stages)
    for (int64_t ns = 1; ns <= nt; ++ns) {
      if (nks[ns - 1] < 2 * cs) break;  // every piece keeps at least two stages
      const int64_t clusters = ns + (nt - ns + cs - 1) / cs;
      if (clusters > cap) continue;
      const int64_t piece = (nks[0] + cs - 1) / cs;
      const int64_t rest = ns < nt ? nks[ns] : 0;
      if (piece > maxst || rest > maxst) continue;
      const int64_t cost = std::max(piece * kCostStage + kCostEpiCluster, rest * kCostStage + kCostEpi);
      if (cost < best.cost || (cost == best.cost && clusters * cs < best.ctas)) {
        best.cs = cs;
        best.T = rest;
        best.cost = cost;
        best.ctas = clusters * cs;
      }
    }
  }
  return best;
}

}  // namespace

int tkb_gemm_split_prepare(tkb_ctx *ctx, tkb_plan *p) {
  const bool cplx = p->dtype == TKB_C128;
  int S = p->slices;
  if (S <= 0) S = 7;
  if (S < 3 || S > SMAX) return tkb_set_error(ctx, TKB_ERR_UNSUPPORTED, "slices must be in 3..7");
  p->slices = S;
  size_t off = 0;
  struct SJob {
    int32_t block, op, r0, kfull, rowc;
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
      const int32_t kfull = cplx ? b.kpad / 2 : b.kpad;
      const int32_t rows_a = cplx ? b.mpad / 2 : b.mpad;  // source rows (complex: row pairs)
      const int32_t ra = b.opA == TKB_OP_N ? 1 : 0, rb = b.opB != TKB_OP_N ? 1 : 0;
      for (int32_t r0 = 0; r0 < rows_a; r0 += 32) sj.push_back({(int32_t)bi, 0, r0, kfull, ra});
      for (int32_t r0 = 0; r0 < b.npad; r0 += 32) sj.push_back({(int32_t)bi, 1, r0, kfull, rb});
    }
    for (int64_t m0 = 0; m0 < M; m0 += PANEL_A)
      for (int64_t n0 = 0; n0 < b.n; n0 += PANEL_B) tiles.push_back({(int32_t)bi, (int32_t)m0, (int32_t)n0, kind});
  }
  // slicing tasks → CTAs: task j gets g_j = min(kSliceCluster, ceil(ntile_j / (8·R))) CTAs (about
  // R warp tiles per warp), tasks are packed first-fit by decreasing g into clusters of
  // kSliceCluster CTAs (the rest idle), and R is the smallest round count whose clusters are
  // all co-resident. 8-K warp tiles when at most two rounds fit one wave, else 16-K tiles.
  std::vector<SliceTask> jobs;
  p->slice_lk = 16;
  if (!sj.empty()) {
    std::stable_sort(sj.begin(), sj.end(), [](const SJob &x, const SJob &y) { return x.kfull > y.kfull; });
    const int wpc = kSliceThreads / 32;
    auto ntile = [&](const SJob &t, int lk) -> int64_t {
      return t.rowc ? t.kfull / lk : (cplx ? 4 : 8) * ((t.kfull + (cplx ? 4 : 8) * lk - 1) / ((cplx ? 4 : 8) * lk));
    };
    // packs with lk and R; false when the clusters exceed cap and `force` is not set
    auto pack = [&](int lk, int R, int64_t cap, bool force) {
      struct Bin {
        int used = 0;
        int64_t len = 0;
        std::vector<std::pair<int, int>> items;  // (job, g)
      };
      std::vector<Bin> bins;
      for (int j = 0; j < (int)sj.size(); ++j) {
        const int64_t nt = ntile(sj[j], lk);
        const int g = (int)std::min<int64_t>(kSliceCluster, std::max<int64_t>(1, (nt + wpc * R - 1) / (wpc * R)));
        size_t bi = 0;
        while (bi < bins.size() && bins[bi].used + g > kSliceCluster) ++bi;
        if (bi == bins.size()) bins.emplace_back();
        bins[bi].items.push_back({j, g});
        bins[bi].used += g;
        bins[bi].len = std::max<int64_t>(bins[bi].len, (nt + wpc * g - 1) / (wpc * g));
      }
      if ((int64_t)bins.size() > cap && !force) return false;
      std::stable_sort(bins.begin(), bins.end(), [](const Bin &x, const Bin &y) { return x.len > y.len; });
      jobs.clear();
      for (const Bin &bn : bins) {
        int rank = 0;
        for (const auto &it : bn.items) {
          const SJob &t = sj[it.first];
          for (int q = 0; q < it.second; ++q) jobs.push_back({t.block, t.op, t.r0, q, it.second, rank});
          rank += it.second;
        }
        for (; rank < kSliceCluster; ++rank) jobs.push_back({0, -1, 0, 0, 1, rank});
      }
      return true;
    };
    const int64_t cap8 = std::max<int64_t>(1, max_slice_clusters(S, cplx, 8, ctx->stream, ctx->num_sms));
    if (pack(8, 1, cap8, false) || pack(8, 2, cap8, false)) {
      p->slice_lk = 8;
    } else {
      const int64_t cap16 = std::max<int64_t>(1, max_slice_clusters(S, cplx, 16, ctx->stream, ctx->num_sms));
      for (int R = 1;; ++R)
        if (pack(16, R, cap16, R >= 64)) break;
    }
  }
  // exponent arrays of every block in one contiguous region (rewritten by every slicing pass)
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
  // tcgen05 tasks: one CTA per SM (the ring fills shared memory). With fewer tiles than SMs,
  // the K loops are cut into pieces of about `target` stages, the smallest target (≥ 4
  // stages) whose task count still fits one wave, so the longest task is as short as possible.
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
    // int32 accumulators stay exact over at most (2^31 − 1)/(S·127²) K positions per task
    const int64_t maxst = std::max<int64_t>(1, (int64_t)2147483647 / ((int64_t)S * 127 * 127) / KSTAGE);
    auto pieces = [&](int64_t nk, int64_t target) {
      return (int)std::max<int64_t>(std::min<int64_t>(8, (nk + target - 1) / target), (nk + maxst - 1) / maxst);
    };
    // cluster plan (partials reduced through distributed shared memory) when it beats both
    // the unsplit plan and the global-memory split plan below
    std::vector<int64_t> nks;
    for (const GTile &t : tiles) nks.push_back(t.kind == 0 ? p->hblocks[t.block].kpad / KSTAGE : 0);
    ClusterPlan cp;
    if (nt < nsm && std::getenv("TKB_SPLIT_REDUCE") == nullptr) cp = plan_clusters(nks, S, maxst, nsm, ctx->stream);
    int64_t target = maxnk;  // no split
    if (nt < nsm) {
      target = std::max<int64_t>(4, (total + nsm - 1) / nsm);
      for (; target < maxnk; ++target) {
        int64_t cnt = 0;
        for (const GTile &t : tiles) cnt += t.kind == 0 ? pieces(p->hblocks[t.block].kpad / KSTAGE, target) : 1;
        if (cnt <= nsm) break;
      }
    }
    // the global-memory split plan's cost in the same model
    int64_t gcost = 0;
    for (const GTile &t : tiles) {
      const int64_t nk = t.kind == 0 ? p->hblocks[t.block].kpad / KSTAGE : 0;
      const int ks = t.kind == 0 ? pieces(nk, target) : 1;
      gcost = std::max<int64_t>(gcost, (nk + ks - 1) / ks * kCostStage +
                                           (ks > 1 ? kCostEpiGlobal + kCostEpiGlobalPiece * (ks - 2) : kCostEpi));
    }
    const bool use_cl = cp.cs > 1 && cp.cost < gcost;
    p->kcluster = use_cl ? cp.cs : 0;
    if (use_cl) {
      // tiles are sorted by decreasing K: split the leading ones, group the rest
      const int cs = cp.cs;
      struct Cl {
        int64_t len;
        SplitTile t[4];
      };
      std::vector<Cl> cls;
      size_t i = 0;
      for (; i < tiles.size() && nks[i] > cp.T; ++i) {
        const GTile &t = tiles[i];
        const int nk = (int)nks[i];
        Cl c;
        c.len = (nk + cs - 1) / cs;
        for (int s = 0; s < cs; ++s) c.t[s] = {t.block, t.m0, t.n0, 0, s * nk / cs, (s + 1) * nk / cs, -1, cs, s, 0};
        cls.push_back(c);
      }
      while (i < tiles.size()) {
        Cl c;
        c.len = nks[i];
        for (int s = 0; s < cs; ++s, ++i) {
          if (i < tiles.size()) {
            const GTile &t = tiles[i];
            c.t[s] = {t.block, t.m0, t.n0, t.kind, 0, (int)nks[i], -1, 1, s, 0};
          } else {
            c.t[s] = {0, 0, 0, 2, 0, 0, -1, 1, s, 0};  // idle
          }
        }
        cls.push_back(c);
      }
      std::stable_sort(cls.begin(), cls.end(), [](const Cl &x, const Cl &y) { return x.len > y.len; });
      for (const Cl &c : cls)
        for (int s = 0; s < cs; ++s) kt.push_back(c.t[s]);
    }
    for (const GTile &t : tiles) {
      if (use_cl) break;
      const int nk = p->hblocks[t.block].kpad / KSTAGE;
      const int ks = t.kind == 0 ? pieces(nk, target) : 1;
      if (ks == 1) {
        kt.push_back({t.block, t.m0, t.n0, t.kind, 0, nk, -1, 1, 0, 0});
      } else {
        const int slot = nslots++;
        for (int s = 0; s < ks; ++s)
          kt.push_back({t.block, t.m0, t.n0, t.kind, s * nk / ks, (s + 1) * nk / ks, slot, ks, s, npart});
        npart += ks;
      }
    }
    if (!use_cl)
      std::stable_sort(kt.begin(), kt.end(), [](const SplitTile &x, const SplitTile &y) {
        return (x.ke - x.kb) > (y.ke - y.kb);
      });
  }
  p->ws_bytes = off;
  p->nstiles = (int64_t)tiles.size();
  p->nkstiles = (int64_t)kt.size();
  // pieces may wait for each other only when every CTA of the launch is resident at once
  p->kspin = (int64_t)kt.size() <= (int64_t)ctx->num_sms ? 1 : 0;
  p->nsjobs = (int)jobs.size();
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
  if (e == cudaSuccess && nslots > 0) {
    const size_t pb = (size_t)npart * 64 * 128 * sizeof(double);
    e = cudaMalloc((void **)&p->part, pb);
    // per slot: arrival counter and completion counter (reset by the last piece)
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->pcnt, 2 * nslots * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->pcnt, 0, 2 * nslots * sizeof(int));
  }
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
