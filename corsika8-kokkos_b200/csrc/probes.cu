// probes.cu — in-run throughput probes for the projection roofline.
//
// The projection is bound by FP64 issue and 64-bit atomics, neither of which
// the HBM/bf16 peak figures cover, so the denominators are measured on the
// same GPU in the same process: dependent-chain-free FP64 and FP32 FMA
// streams, and 64-bit atomic adds to distinct shared and global addresses.
#include <cuda_runtime.h>

#include "../../include/c8radio.h"

namespace {

constexpr int kChains = 8;

template <class T>
__global__ void __launch_bounds__(256) fma_stream(T* sink, int iterations, T b, T c) {
  T acc[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) acc[k] = static_cast<T>(threadIdx.x + k);
  for (int i = 0; i < iterations; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc[k] = fma(acc[k], b, c);
  }
  T total = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) total += acc[k];
  if (total == static_cast<T>(-1.2345)) *sink = total;  // keeps the chains live
}

__global__ void __launch_bounds__(256) shared_atomics(unsigned long long* sink, int iterations) {
  __shared__ unsigned long long window[4096];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) window[i] = 0;
  __syncthreads();
  unsigned const base = threadIdx.x * 13u;
  for (int i = 0; i < iterations; ++i) atomicAdd(&window[(base + i * 97u) & 4095u], 1ull);
  __syncthreads();
  if (threadIdx.x == 0 && window[0] == 0xdeadbeefull) *sink = window[1];
}

__global__ void __launch_bounds__(256) global_atomics(unsigned long long* rows, unsigned long long mask,
                                                      int iterations) {
  unsigned long long const base =
      (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) * 7919ull;
  for (int i = 0; i < iterations; ++i)
    atomicAdd(&rows[(base + static_cast<unsigned long long>(i) * 104729ull) & mask], 1ull);
}

template <class F>
float time_ms(F&& launch) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch();  // warm
  cudaEventRecord(a);
  launch();
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

}  // namespace

extern "C" int c8r_probe_peaks(c8r_peaks* out) {
  if (!out) return C8R_INVALID_ARGUMENT;
  int device = 0, sms = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return C8R_CUDA_ERROR;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* dsink = nullptr;
  unsigned long long* rows = nullptr;
  unsigned long long const global_values = 1ull << 24;  // 128 MiB of counters (> L2)
  if (cudaMalloc(&dsink, 64) != cudaSuccess) return C8R_BAD_ALLOC;
  if (cudaMalloc(&rows, global_values * sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(dsink);
    return C8R_BAD_ALLOC;
  }
  cudaMemset(rows, 0, global_values * sizeof(unsigned long long));
  int const blocks = sms * 8, threads = 256, iterations = 4096;
  double const fma_ops = 2.0 * kChains * static_cast<double>(iterations) * blocks * threads;
  float ms = time_ms([&] { fma_stream<double><<<blocks, threads>>>(dsink, iterations, 0.999999, 1e-9); });
  out->fp64_flops = fma_ops / (ms * 1e-3);
  ms = time_ms([&] {
    fma_stream<float><<<blocks, threads>>>(reinterpret_cast<float*>(dsink), iterations, 0.999999f, 1e-9f);
  });
  out->fp32_flops = fma_ops / (ms * 1e-3);
  int const atom_iterations = 2048;
  ms = time_ms([&] {
    shared_atomics<<<blocks, threads>>>(reinterpret_cast<unsigned long long*>(dsink), atom_iterations);
  });
  out->shared_atomics_per_s = static_cast<double>(atom_iterations) * blocks * threads / (ms * 1e-3);
  int const global_iterations = 256;
  ms = time_ms([&] { global_atomics<<<blocks, threads>>>(rows, global_values - 1, global_iterations); });
  out->global_atomics_per_s = static_cast<double>(global_iterations) * blocks * threads / (ms * 1e-3);
  cudaError_t const err = cudaGetLastError();
  cudaFree(rows);
  cudaFree(dsink);
  return err == cudaSuccess ? C8R_OK : C8R_CUDA_ERROR;
}
