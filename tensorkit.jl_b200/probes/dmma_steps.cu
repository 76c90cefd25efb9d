// Throughput probe: which part of a plain FP64 GEMM step slows DMMA issue on B200. One CTA (or two)
// per SM of 128 or 256 threads, each warp a 32×32 tile (2×4 m16n8k8 accumulators); a "step" is 8
// DMMA per warp (one K sub-step of 8) on a 16-wide ring slot of 64×64 operand tiles.
//   mode 0: fragments in registers (2 a × 4 b, varied)
//   mode 2: fragments read from shared memory, a barrier per step
//   mode 3: mode 2 plus the refill of a 16 KB stage two steps ahead by per-thread 16-byte cp.async
//           (the plain kernel's ring: wait, barrier, copies, then DMMA)
//   mode 4: mode 2 plus the refill by 80 bulk copies (one per tile column) on an mbarrier
//   mode 5: mode 3 with the copies issued after the step's DMMA
// Every copy reads a 32 KB source that stays in L2; every wait is bounded.
// Build and run: nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o dmma_steps dmma_steps.cu && ./dmma_steps
#include <cstdio>
#include <cuda_runtime.h>

__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

struct Sm {
  double A[3][16][68];
  double B[3][64][20];
};

template <int MODE>
__global__ void step_kernel(double *out, const double *src, int steps) {
  extern __shared__ __align__(16) unsigned char raw[];
  Sm &s = *reinterpret_cast<Sm *>(raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = (warp >> 1) & 1, kg = (warp >> 2) & 1;
  const int g = lane >> 2, t = lane & 3;
  __shared__ __align__(8) unsigned long long full[3];
  __shared__ int bad;
  if (tid == 0) {
    bad = 0;
    for (int i = 0; i < 3; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"((unsigned)__cvta_generic_to_shared(&full[i])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int e = tid; e < 3 * 16 * 68; e += blockDim.x) (&s.A[0][0][0])[e] = 1e-3 * (e % 17);
  for (int e = tid; e < 3 * 64 * 20; e += blockDim.x) (&s.B[0][0][0])[e] = 1e-3 * (e % 13);
  __syncthreads();
  double acc[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) acc[q] = 0.0;
  double af[2][4], bf[4][2];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int q = 0; q < 4; ++q) af[mi][q] = 1e-3 * (mi * 4 + q + lane);
#pragma unroll
  for (int ni = 0; ni < 4; ++ni) bf[ni][0] = bf[ni][1] = 1e-3 * (ni + lane);
  const int kk = 8 * kg;
  if (MODE == 3 || MODE == 5) {
    for (int p = 0; p < 2; ++p) {
      for (int e = tid; e < 16 * 64 / 2; e += blockDim.x) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(&s.A[p][e / 32][2 * (e % 32)]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 2 * e));
      }
      asm volatile("cp.async.commit_group;\n" ::);
    }
  }
  if (MODE == 4 && tid == 0) {
    // the first two slots are "filled" by an arrival without bytes
    for (int p = 0; p < 2; ++p)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"((unsigned)__cvta_generic_to_shared(&full[p])) : "memory");
  }
  for (int it = 0; it < steps; ++it) {
    const int st = it % 3;
    if (MODE == 5) {
      asm volatile("cp.async.wait_group 1;\n" ::);
      __syncthreads();
    }
    if (MODE == 3) {
      asm volatile("cp.async.wait_group 1;\n" ::);
      __syncthreads();
      const int nx = (it + 2) % 3;
      for (int e = tid; e < 16 * 64 / 2; e += blockDim.x) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(&s.A[nx][e / 32][2 * (e % 32)]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 2 * e));
      }
      for (int e = tid; e < 16 * 64 / 2; e += blockDim.x) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(&s.B[nx][e / 8][2 * (e % 8)]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 1024 + 2 * e));
      }
      asm volatile("cp.async.commit_group;\n" ::);
    } else if (MODE == 4) {
      // wait for this step's slot (bounded), then refill the slot two steps ahead with bulk copies
      const unsigned fb = (unsigned)__cvta_generic_to_shared(&full[st]);
      const unsigned par = (unsigned)((it / 3) & 1);
      unsigned ok = 0;
      for (int n = 0; n < (1 << 22) && !ok; ++n)
        asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok) : "r"(fb), "r"(par) : "memory");
      if (!ok) bad = 1;
      __syncthreads();
      if (warp == 0 && it + 2 < steps) {
        const int nx = (it + 2) % 3;
        const unsigned nb = (unsigned)__cvta_generic_to_shared(&full[nx]);
        if (lane == 0) asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(nb), "r"(16384u) : "memory");
        __syncwarp();
        for (int c = lane; c < 16 + 64; c += 32) {
          unsigned d; const double *g; unsigned sz;
          if (c < 16) { d = (unsigned)__cvta_generic_to_shared(&s.A[nx][c][0]); g = src + 64 * c; sz = 512; }
          else { d = (unsigned)__cvta_generic_to_shared(&s.B[nx][c - 16][0]); g = src + 1024 + 16 * (c - 16); sz = 128; }
          asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                       ::"r"(d), "l"(g), "r"(sz), "r"(nb) : "memory");
        }
      }
    } else if (MODE >= 2) {
      __syncthreads();
    }
    if (MODE >= 1) {
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
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) dmma16(*reinterpret_cast<double(*)[4]>(&acc[(mi * 4 + ni) * 4]), af[mi], bf[ni]);
    if (MODE == 5) {
      const int nx = (it + 2) % 3;
      for (int e = tid; e < 16 * 64 / 2; e += blockDim.x) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(&s.A[nx][e / 32][2 * (e % 32)]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 2 * e));
      }
      for (int e = tid; e < 16 * 64 / 2; e += blockDim.x) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(&s.B[nx][e / 8][2 * (e % 8)]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 1024 + 2 * e));
      }
      asm volatile("cp.async.commit_group;\n" ::);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
  // mode 4 issues a stage only while it + 2 < steps, so every bulk copy has been waited for here
  double sum = bad ? 1e300 : 0;
#pragma unroll
  for (int q = 0; q < 32; ++q) sum += acc[q];
  out[blockIdx.x * blockDim.x + tid] = sum;
}

template <int MODE>
void run(int sms, int threads, int per_sm, double *out, const double *src) {
  const int steps = 2000, blocks = sms * per_sm;
  auto k = step_kernel<MODE>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Sm));
  k<<<blocks, threads, sizeof(Sm)>>>(out, src, 10);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  k<<<blocks, threads, sizeof(Sm)>>>(out, src, steps);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms;
  cudaEventElapsedTime(&ms, a, b);
  const double dmma_per_smsp = (double)steps * (threads / 32) * 8 * per_sm / 4;
  const double fl = 2.0 * 1024 * 8 * steps * (double)(threads / 32) * blocks;
  printf("mode %d threads %3d ctas/SM %d: %.3f ms %6.2f TF/s  %.0f ns per step  %.1f cycles/DMMA/SMSP at 1965 MHz\n",
         MODE, threads, per_sm, ms, fl / ms / 1e9, ms * 1e6 / steps, ms * 1e-3 * 1.965e9 / dmma_per_smsp);
}

int main() {
  int sms;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  double *out, *src;
  cudaMalloc(&out, (size_t)sms * 4 * 256 * sizeof(double));
  cudaMalloc(&src, 4096 * sizeof(double));  // reads stay below 2048 + 1024 doubles
  cudaMemset(src, 0, 4096 * sizeof(double));
  for (int threads : {128, 256})
    for (int per_sm : {1, 2}) {
      run<0>(sms, threads, per_sm, out, src);
      run<2>(sms, threads, per_sm, out, src);
      run<3>(sms, threads, per_sm, out, src);
      run<4>(sms, threads, per_sm, out, src);
      run<5>(sms, threads, per_sm, out, src);
    }
  cudaError_t e = cudaDeviceSynchronize();
  printf("status %s\n", cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
