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
// Launches: slice pass (all operand rows of all blocks, one warp per row) + product pass
// (persistent CTAs over a cost-ordered tile queue, 64×64 output tiles).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "tkb_internal.h"

namespace {

constexpr int SBM = 64, SBN = 64, SBK = 32;  // SBK: bytes (int8 elements) of K per step
constexpr int SPITCH = 48;                    // smem row pitch in bytes: conflict-free frags
constexpr int SMAX = 7;

struct SliceJob {
  int32_t block;
  int32_t operand;  // 0 = rows of op(A), 1 = columns of op(B)
};

struct CDbl {
  double x, y;
};

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

// One warp per logical row of every operand of every block (rows enumerated through the
// row_begin prefix sums, padding rows included so the padded slices are zero-filled).
__global__ void __launch_bounds__(256)
    slice_kernel(const GBlock *__restrict__ blocks, const int64_t *__restrict__ row_begin,
                 const SliceJob *__restrict__ jobs, int njobs, int64_t nrows, int S, int cplx,
                 const double *__restrict__ A, const double *__restrict__ B, int8_t *ws) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t row = wid; row < nrows; row += nw) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (row_begin[mid] <= row) lo = mid; else hi = mid - 1;
    }
    const SliceJob job = jobs[lo];
    const GBlock &b = blocks[job.block];
    const int64_t r = row - row_begin[lo];
    const int64_t Mlog = job.operand == 0 ? (cplx ? 2 * b.m : b.m) : b.n;
    const int64_t Klog = cplx ? 2 * b.k : b.k;
    const int64_t rows_pad = job.operand == 0 ? b.mpad : b.npad;
    const int64_t kpad = b.kpad;
    int8_t *base = ws + (job.operand == 0 ? b.wsA : b.wsB);
    int32_t *expo = reinterpret_cast<int32_t *>(ws + (job.operand == 0 ? b.wsEA : b.wsEB));
    const double *X = job.operand == 0 ? A : B;
    const bool valid = r < Mlog;
    double mx = 0.0;
    if (valid) {
      for (int64_t l = lane; l < Klog; l += 32)
        mx = fmax(mx, fabs(op_elem(b, job.operand, cplx, X, r, l)));
      if (cplx && job.operand == 0) {  // a complex row pair shares one exponent
        for (int64_t l = lane; l < Klog; l += 32)
          mx = fmax(mx, fabs(op_elem(b, job.operand, cplx, X, r ^ 1, l)));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);  // mx < 2^e
    if (lane == 0) expo[r] = e;
    for (int64_t l = lane; l < kpad; l += 32) {
      double x = 0.0;
      if (valid && l < Klog) x = ldexp(op_elem(b, job.operand, cplx, X, r, l), -e);
      for (int s = 0; s < S; ++s) {
        x *= 128.0;
        const double q = trunc(x);
        x -= q;
        base[(int64_t)s * rows_pad * kpad + r * kpad + l] = (int8_t)q;
      }
    }
    (void)rows_pad;
  }
}

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
__device__ __forceinline__ void load_stage(int8_t *As, int8_t *Bs, const GBlock &b,
                                           const int8_t *ws, int64_t m0, int64_t n0, int64_t k0) {
  // per slice: 64 rows x 32 bytes = 128 chunks of 16 bytes for each operand
  for (int c = threadIdx.x; c < 2 * S * 128; c += blockDim.x) {
    const int op = c / (S * 128);
    const int rem = c % (S * 128);
    const int s = rem / 128, q = rem % 128;
    const int row = q >> 1, half = q & 1;
    if (op == 0) {
      const int8_t *g = ws + b.wsA + ((int64_t)s * b.mpad + m0 + row) * b.kpad + k0 + half * 16;
      cp_async16(As + (s * SBM + row) * SPITCH + half * 16, g);
    } else {
      const int8_t *g = ws + b.wsB + ((int64_t)s * b.npad + n0 + row) * b.kpad + k0 + half * 16;
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
    const int64_t m0 = tile.m0, n0 = tile.n0;
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
    // epilogue: recombine the diagonals in FP64, smallest weight first
    const int32_t *eA = reinterpret_cast<const int32_t *>(ws + b.wsEA);
    const int32_t *eB = reinterpret_cast<const int32_t *>(ws + b.wsEB);
    const int64_t Mreal = cplx ? 2 * b.m : b.m;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int64_t i = m0 + wm * 32 + mt * 16 + g + hr * 8;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
#pragma unroll
          for (int hc = 0; hc < 2; ++hc) {
            const int64_t j = n0 + wn * 16 + nt * 8 + 2 * tig + hc;
            double v = 0.0;
            if (tile.kind == 0) {
#pragma unroll
              for (int d = S - 1; d >= 0; --d)
                v += ldexp((double)acc[d][mt][nt][hr * 2 + hc], -7 * (d + 2));
              const int ei = (i < Mreal) ? eA[i] : 0;
              const int ej = (j < b.n) ? eB[j] : 0;
              v = ldexp(v, ei + ej);
            }
            if (!cplx) {
              if (i < b.m && j < b.n) {
                double *p = C + b.offC + i + j * b.ldc;
                double r = alpha.x * v;
                if (!bz) r = fma(beta.x, *p, r);
                *p = r;
              }
            } else {
              const double w = __shfl_xor_sync(0xffffffffu, v, 4);  // partner row (g ^ 1)
              if (!(g & 1) && i < Mreal && j < b.n) {
                const double vr = v, vi = w;
                double2 *p = reinterpret_cast<double2 *>(C) + b.offC + (i >> 1) + j * b.ldc;
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

template <int S>
int launch_split(tkb_ctx *ctx, const tkb_plan *p, void *C, CDbl a, CDbl b) {
  const size_t smem = 2 * (size_t)(2 * S * SBM * SPITCH);
  auto k = gemm_split_mma_kernel<S>;
  TKB_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>(p->nstiles, (int64_t)ctx->num_sms * 2);
  k<<<grid, 256, smem, ctx->stream>>>(p->blocks, p->stiles, (int)p->nstiles, ctx->counters,
                                      (const int8_t *)ctx->ws, p->dtype == TKB_C128 ? 1 : 0,
                                      (double *)C, a, b);
  ctx->launches++;
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
  std::vector<int64_t> row_begin;
  std::vector<GTile> tiles;
  int64_t nrows = 0;
  for (size_t bi = 0; bi < p->hblocks.size(); ++bi) {
    GBlock &b = p->hblocks[bi];
    const int64_t M = cplx ? 2 * b.m : b.m;
    const int64_t K = cplx ? 2 * b.k : b.k;
    b.mpad = (int32_t)roundup(std::max<int64_t>(M, 1), SBM);
    b.npad = (int32_t)roundup(std::max<int64_t>(b.n, 1), SBN);
    b.kpad = (int32_t)roundup(std::max<int64_t>(K, 1), SBK);
    if (b.m == 0 || b.n == 0) continue;
    b.wsA = (int64_t)off;
    off += (size_t)S * b.mpad * b.kpad;
    b.wsB = (int64_t)off;
    off += (size_t)S * b.npad * b.kpad;
    off = roundup((int64_t)off, 256);
    b.wsEA = (int64_t)off;
    off += (size_t)b.mpad * 4;
    b.wsEB = (int64_t)off;
    off += (size_t)b.npad * 4;
    off = roundup((int64_t)off, 256);
    const int kind = b.k > 0 ? 0 : 1;
    if (kind == 0) {
      jobs.push_back({(int32_t)bi, 0});
      row_begin.push_back(nrows);
      nrows += b.mpad;
      jobs.push_back({(int32_t)bi, 1});
      row_begin.push_back(nrows);
      nrows += b.npad;
    }
    for (int64_t m0 = 0; m0 < M; m0 += SBM)
      for (int64_t n0 = 0; n0 < b.n; n0 += SBN) tiles.push_back({(int32_t)bi, (int32_t)m0, (int32_t)n0, kind});
  }
  std::stable_sort(tiles.begin(), tiles.end(), [&](const GTile &x, const GTile &y) {
    return p->hblocks[x.block].kpad > p->hblocks[y.block].kpad;
  });
  p->ws_bytes = off;
  p->nstiles = (int64_t)tiles.size();
  p->nsjobs = (int)jobs.size();
  p->nsrows = nrows;
  cudaError_t e = cudaSuccess;
  if (!tiles.empty()) {
    e = cudaMalloc((void **)&p->stiles, tiles.size() * sizeof(GTile));
    if (e == cudaSuccess) e = cudaMemcpy(p->stiles, tiles.data(), tiles.size() * sizeof(GTile), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !jobs.empty()) {
    e = cudaMalloc(&p->sjobs, jobs.size() * sizeof(SliceJob));
    if (e == cudaSuccess) e = cudaMemcpy(p->sjobs, jobs.data(), jobs.size() * sizeof(SliceJob), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->srow_begin, row_begin.size() * 8);
    if (e == cudaSuccess) e = cudaMemcpy(p->srow_begin, row_begin.data(), row_begin.size() * 8, cudaMemcpyHostToDevice);
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
  const int cplx = p->dtype == TKB_C128 ? 1 : 0;
  if (p->nsrows > 0) {
    const int64_t warps = p->nsrows;
    const int grid = (int)std::min<int64_t>((warps + 7) / 8, (int64_t)ctx->num_sms * 16);
    slice_kernel<<<grid, 256, 0, ctx->stream>>>(p->blocks, p->srow_begin,
                                                (const SliceJob *)p->sjobs, p->nsjobs, p->nsrows,
                                                p->slices, cplx, (const double *)A,
                                                (const double *)B, (int8_t *)ctx->ws);
    ctx->launches++;
    TKB_CUDA_TRY(ctx, cudaGetLastError());
  }
  CDbl a{alpha.re, alpha.im}, b{beta.re, beta.im};
  int rc;
  switch (p->slices) {
    case 3: rc = launch_split<3>(ctx, p, C, a, b); break;
    case 4: rc = launch_split<4>(ctx, p, C, a, b); break;
    case 5: rc = launch_split<5>(ctx, p, C, a, b); break;
    case 6: rc = launch_split<6>(ctx, p, C, a, b); break;
    default: rc = launch_split<7>(ctx, p, C, a, b); break;
  }
  if (rc != TKB_OK) return rc;
  TKB_CUDA_TRY(ctx, cudaGetLastError());
  return TKB_OK;
}
