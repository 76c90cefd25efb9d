// FP64 throughput probe on B200: DFMA chains against m16n8k8 and m8n8k4 DMMA with independent
// accumulators, 8 to 64 warps per SM, all operands in registers (the pipe peaks behind the plain
// GEMM's roofline). Build and run:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o fp64rate fp64rate.cu && ./fp64rate
#include <cstdio>
#include <cuda_runtime.h>

__global__ void dfma_kernel(double *out, int iters, double x) {
  double c[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) c[i] = x * (i + 1);
  const double a = x * 0.999, b = 1.0 + 1e-9 * threadIdx.x;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 16; ++i) c[i] = fma(c[i], b, a);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) s += c[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
__device__ __forceinline__ void dmma4(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int NACC>
__global__ void dmma16_kernel(double *out, int iters, double x) {
  double c[NACC][4];
#pragma unroll
  for (int i = 0; i < NACC; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) c[i][q] = 0.0;
  double a[4] = {x, x * 0.5, x * 0.25, x * 0.125};
  double b[2] = {1e-3 * threadIdx.x, 2e-3};
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < NACC; ++i) dmma16(c[i], a, b);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < NACC; ++i) s += c[i][0] + c[i][1] + c[i][2] + c[i][3];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <int NACC>
__global__ void dmma4_kernel(double *out, int iters, double x) {
  double c[NACC][2];
#pragma unroll
  for (int i = 0; i < NACC; ++i) c[i][0] = c[i][1] = 0.0;
  const double a = x, b = 1e-3 * threadIdx.x;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < NACC; ++i) dmma4(c[i][0], c[i][1], a, b);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < NACC; ++i) s += c[i][0] + c[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename F>
float timeit(F f) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  f();
  cudaDeviceSynchronize();
  cudaEventRecord(a);
  for (int r = 0; r < 5; ++r) f();
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms;
  cudaEventElapsedTime(&ms, a, b);
  return ms / 5;
}

int main() {
  int sms;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const int maxblocks = sms * 8, threads = 256;
  double *out;
  cudaMalloc(&out, (size_t)maxblocks * threads * sizeof(double));
  const int iters = 4096;
  for (int per_sm : {1, 2, 4, 8}) {
    const int blocks = sms * per_sm;
    float ms = timeit([&] { dfma_kernel<<<blocks, threads>>>(out, iters, 1.0); });
    double fl = 2.0 * 16 * iters * (double)blocks * threads;
    printf("DFMA    warps/SM %2d: %.3f ms  %.2f TFLOP/s\n", per_sm * 8, ms, fl / ms / 1e9);
  }
  for (int per_sm : {1, 2, 4, 8}) {
    const int blocks = sms * per_sm;
    float ms = timeit([&] { dmma16_kernel<8><<<blocks, threads>>>(out, iters / 4, 1.0); });
    double fl = 2.0 * 1024 * 8 * (iters / 4) * (double)blocks * (threads / 32);
    printf("DMMA16x8 warps/SM %2d: %.3f ms  %.2f TFLOP/s\n", per_sm * 8, ms, fl / ms / 1e9);
  }
  for (int per_sm : {1, 2, 4}) {
    const int blocks = sms * per_sm;
    float ms = timeit([&] { dmma16_kernel<16><<<blocks, threads>>>(out, iters / 8, 1.0); });
    double fl = 2.0 * 1024 * 16 * (iters / 8) * (double)blocks * (threads / 32);
    printf("DMMA16x16 warps/SM %2d: %.3f ms  %.2f TFLOP/s\n", per_sm * 8, ms, fl / ms / 1e9);
  }
  for (int per_sm : {1, 2, 4, 8}) {
    const int blocks = sms * per_sm;
    float ms = timeit([&] { dmma4_kernel<8><<<blocks, threads>>>(out, iters / 2, 1.0); });
    double fl = 2.0 * 256 * 8 * (iters / 2) * (double)blocks * (threads / 32);
    printf("DMMA4x8 warps/SM %2d: %.3f ms  %.2f TFLOP/s\n", per_sm * 8, ms, fl / ms / 1e9);
  }
  cudaError_t e = cudaGetLastError();
  printf("status %s\n", cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
