// Plain FP64 / ComplexF64 grouped block GEMM: one persistent launch for all coupled-sector
// blocks of a TensorKit mul! (src/tensors/linalg.jl:330-370), tiles taken from a
// cost-ordered device work queue (largest k first).
//
// Tensor path: FP64 DMMA (mma.sync.m8n8k4.f64). tcgen05 has no f64 kind, so the
// double-precision tensor pipe is reached through DMMA; the split-precision path
// (gemm_split.cu) is the tcgen05 one.
//
// CTA tile 64x64x16, 4 warps in a 2x2 grid (each 32x32 = 4x4 DMMA tiles), operands
// double-buffered in shared memory with 8-byte cp.async (zero-filled outside the block,
// so any lda/offset parity works). Complex blocks keep separate re/im planes and issue
// four real DMMA per fragment pair.
#include <algorithm>
#include <cstring>

#include "tkb_internal.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 16;
constexpr int APAD = 4, BPAD = 4;

struct CDbl {
  double x, y;
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// ---- real ----------------------------------------------------------------------------
struct SmemR {
  double A[2][BK][BM + APAD];
  double B[2][BN][BK + BPAD];
};

__device__ __forceinline__ void load_tiles_r(SmemR &s, int buf, const GBlock &b, const double *A,
                                             const double *B, int64_t m0, int64_t n0, int64_t k0) {
  const int tid = threadIdx.x;
  // A tile: op(A) rows m0.., cols k0..
  if (b.opA == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BM * BK) / 128; ++r) {
      const int e = tid + r * 128;
      const int i = e % BM, l = e / BM;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      const double *p = A + b.offA + (ok ? gi + gl * b.lda : 0);
      cp_async8(&s.A[buf][l][i], p, ok);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BM * BK) / 128; ++r) {
      const int e = tid + r * 128;
      const int l = e % BK, i = e / BK;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      const double *p = A + b.offA + (ok ? gl + gi * b.lda : 0);
      cp_async8(&s.A[buf][l][i], p, ok);
    }
  }
  if (b.opB == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BN * BK) / 128; ++r) {
      const int e = tid + r * 128;
      const int l = e % BK, j = e / BK;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      const double *p = B + b.offB + (ok ? gl + gj * b.ldb : 0);
      cp_async8(&s.B[buf][j][l], p, ok);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BN * BK) / 128; ++r) {
      const int e = tid + r * 128;
      const int j = e % BN, l = e / BN;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      const double *p = B + b.offB + (ok ? gj + gl * b.ldb : 0);
      cp_async8(&s.B[buf][j][l], p, ok);
    }
  }
}

__global__ void __launch_bounds__(128)
    gemm_f64_kernel(const GBlock *__restrict__ blocks, const GTile *__restrict__ tiles, int ntiles,
                    int *counters, double *__restrict__ C, const double *__restrict__ A,
                    const double *__restrict__ B, double alpha, double beta) {
  __shared__ __align__(16) SmemR s;
  __shared__ int next_tile;
  pdl_wait();  // operands, output and the work-queue counters belong to earlier kernels too
  pdl_trigger();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  while (true) {
    if (threadIdx.x == 0) next_tile = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int ti = next_tile;
    __syncthreads();
    if (ti >= ntiles) break;
    const GTile tile = tiles[ti];
    const GBlock b = blocks[tile.block];
    const int64_t m0 = tile.m0, n0 = tile.n0;
    double acc[4][4][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    const int64_t nk = (b.k + BK - 1) / BK;
    if (nk > 0) {
      load_tiles_r(s, 0, b, A, B, m0, n0, 0);
      cp_async_commit();
      for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) {
          load_tiles_r(s, buf ^ 1, b, A, B, m0, n0, (kt + 1) * BK);
          cp_async_commit();
          cp_async_wait_1();
        } else {
          cp_async_wait_all();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
          double af[4], bf[4];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) af[mi] = s.A[buf][kk + t][wm * 32 + mi * 8 + g];
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) bf[ni] = s.B[buf][wn * 32 + ni * 8 + g][kk + t];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
        }
        __syncthreads();
      }
    }
    // epilogue: C = α·acc + β·C
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int64_t i = m0 + wm * 32 + mi * 8 + g;
      if (i >= b.m) continue;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t j = n0 + wn * 32 + ni * 8 + 2 * t + h;
          if (j >= b.n) continue;
          double *p = C + b.offC + i + j * b.ldc;
          double r = alpha * acc[mi][ni][h];
          if (beta != 0.0) r = fma(beta, *p, r);
          *p = r;
        }
      }
    }
  }
  // self-resetting queue: the last CTA out zeroes the counters for the next launch
  if (threadIdx.x == 0) {
    __threadfence();
    const int done = atomicAdd(&counters[1], 1);
    if (done == (int)gridDim.x - 1) {
      atomicExch(&counters[0], 0);
      atomicExch(&counters[1], 0);
      __threadfence();
    }
  }
}

// ---- complex ---------------------------------------------------------------------------
struct SmemC {
  double Ar[2][BK][BM + APAD];
  double Ai[2][BK][BM + APAD];
  double Br[2][BN][BK + BPAD];
  double Bi[2][BN][BK + BPAD];
};

__device__ __forceinline__ void load_tiles_c(SmemC &s, int buf, const GBlock &b, const double2 *A,
                                             const double2 *B, int64_t m0, int64_t n0, int64_t k0) {
  const int tid = threadIdx.x;  // 256 threads
  const double *Ad = reinterpret_cast<const double *>(A);
  const double *Bd = reinterpret_cast<const double *>(B);
  if (b.opA == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BM * BK) / 256; ++r) {
      const int e = tid + r * 256;
      const int i = e % BM, l = e / BM;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      const int64_t idx = ok ? b.offA + gi + gl * b.lda : 0;
      cp_async8(&s.Ar[buf][l][i], Ad + 2 * idx, ok);
      cp_async8(&s.Ai[buf][l][i], Ad + 2 * idx + 1, ok);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BM * BK) / 256; ++r) {
      const int e = tid + r * 256;
      const int l = e % BK, i = e / BK;
      const int64_t gi = m0 + i, gl = k0 + l;
      const bool ok = gi < b.m && gl < b.k;
      const int64_t idx = ok ? b.offA + gl + gi * b.lda : 0;
      cp_async8(&s.Ar[buf][l][i], Ad + 2 * idx, ok);
      cp_async8(&s.Ai[buf][l][i], Ad + 2 * idx + 1, ok);
    }
  }
  if (b.opB == TKB_OP_N) {
#pragma unroll
    for (int r = 0; r < (BN * BK) / 256; ++r) {
      const int e = tid + r * 256;
      const int l = e % BK, j = e / BK;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      const int64_t idx = ok ? b.offB + gl + gj * b.ldb : 0;
      cp_async8(&s.Br[buf][j][l], Bd + 2 * idx, ok);
      cp_async8(&s.Bi[buf][j][l], Bd + 2 * idx + 1, ok);
    }
  } else {
#pragma unroll
    for (int r = 0; r < (BN * BK) / 256; ++r) {
      const int e = tid + r * 256;
      const int j = e % BN, l = e / BN;
      const int64_t gl = k0 + l, gj = n0 + j;
      const bool ok = gl < b.k && gj < b.n;
      const int64_t idx = ok ? b.offB + gj + gl * b.ldb : 0;
      cp_async8(&s.Br[buf][j][l], Bd + 2 * idx, ok);
      cp_async8(&s.Bi[buf][j][l], Bd + 2 * idx + 1, ok);
    }
  }
}

__global__ void __launch_bounds__(256)
    gemm_c128_kernel(const GBlock *__restrict__ blocks, const GTile *__restrict__ tiles, int ntiles,
                     int *counters, double2 *__restrict__ C, const double2 *__restrict__ A,
                     const double2 *__restrict__ B, CDbl alpha, CDbl beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemC &s = *reinterpret_cast<SmemC *>(smem_raw);
  __shared__ int next_tile;
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;  // 8 warps: 2 (m) x 4 (n)
  const int wm = warp & 1, wn = warp >> 1;                      // warp tile 32 x 16
  const int g = lane >> 2, t = lane & 3;
  const bool bz = beta.x == 0.0 && beta.y == 0.0;
  while (true) {
    if (threadIdx.x == 0) next_tile = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int ti = next_tile;
    __syncthreads();
    if (ti >= ntiles) break;
    const GTile tile = tiles[ti];
    const GBlock b = blocks[tile.block];
    // conjugation of an operand flips the sign of its imaginary plane
    const double sa = (b.opA == TKB_OP_C) ? -1.0 : 1.0;
    const double sb = (b.opB == TKB_OP_C) ? -1.0 : 1.0;
    const int64_t m0 = tile.m0, n0 = tile.n0;
    double ar[4][2][2], ai[4][2][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) ar[mi][ni][0] = ar[mi][ni][1] = ai[mi][ni][0] = ai[mi][ni][1] = 0.0;
    const int64_t nk = (b.k + BK - 1) / BK;
    if (nk > 0) {
      load_tiles_c(s, 0, b, A, B, m0, n0, 0);
      cp_async_commit();
      for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) {
          load_tiles_c(s, buf ^ 1, b, A, B, m0, n0, (kt + 1) * BK);
          cp_async_commit();
          cp_async_wait_1();
        } else {
          cp_async_wait_all();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
          double fr[4], fi[4], fin[4], gr[2], gi[2];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) {
            fr[mi] = s.Ar[buf][kk + t][wm * 32 + mi * 8 + g];
            fi[mi] = sa * s.Ai[buf][kk + t][wm * 32 + mi * 8 + g];
            fin[mi] = -fi[mi];
          }
#pragma unroll
          for (int ni = 0; ni < 2; ++ni) {
            gr[ni] = s.Br[buf][wn * 16 + ni * 8 + g][kk + t];
            gi[ni] = sb * s.Bi[buf][wn * 16 + ni * 8 + g][kk + t];
          }
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) {
              dmma(ar[mi][ni][0], ar[mi][ni][1], fr[mi], gr[ni]);
              dmma(ar[mi][ni][0], ar[mi][ni][1], fin[mi], gi[ni]);
              dmma(ai[mi][ni][0], ai[mi][ni][1], fr[mi], gi[ni]);
              dmma(ai[mi][ni][0], ai[mi][ni][1], fi[mi], gr[ni]);
            }
        }
        __syncthreads();
      }
    }
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
          const double vr = ar[mi][ni][h], vi = ai[mi][ni][h];
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
  if (threadIdx.x == 0) {
    __threadfence();
    const int done = atomicAdd(&counters[1], 1);
    if (done == (int)gridDim.x - 1) {
      atomicExch(&counters[0], 0);
      atomicExch(&counters[1], 0);
      __threadfence();
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

int tkb_gemm_launch(tkb_ctx *ctx, const tkb_plan *p, void *C, const void *A, const void *B,
                    tkb_scalar alpha, tkb_scalar beta) {
  if (p->ntiles == 0) return TKB_OK;
  if (p->dtype == TKB_F64) {
    if (alpha.im != 0.0 || beta.im != 0.0)
      return tkb_set_error(ctx, TKB_ERR_ARG, "complex scalar with real data");
    const int grid = (int)std::min<int64_t>(p->ntiles, (int64_t)ctx->num_sms * 4);
    TKB_CUDA_TRY(ctx, launch_pdl(gemm_f64_kernel, dim3(grid), dim3(128), 0, ctx->stream, p->blocks, p->tiles,
                                 (int)p->ntiles, ctx->counters, (double *)C, (const double *)A,
                                 (const double *)B, alpha.re, beta.re));
  } else {
    const int grid = (int)std::min<int64_t>(p->ntiles, (int64_t)ctx->num_sms * 2);
    const size_t smem = sizeof(SmemC);
    TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(gemm_c128_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TKB_CUDA_TRY(ctx, launch_pdl(gemm_c128_kernel, dim3(grid), dim3(256), smem, ctx->stream, p->blocks, p->tiles,
                                 (int)p->ntiles, ctx->counters, (double2 *)C, (const double2 *)A,
                                 (const double2 *)B, CDbl{alpha.re, alpha.im}, CDbl{beta.re, beta.im}));
  }
  ctx->launches++;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}
