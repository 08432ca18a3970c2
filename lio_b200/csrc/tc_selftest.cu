// Self-test of the tcgen05 int8 GEMM primitive (umma.cuh): D[128 x N] =
// A[128 x K] * B[N x K]^T with exact int32 accumulation in TMEM. Exposed as a
// C entry point so the GPU tests can check the descriptor encodings and the
// TMEM read-back layout against an exact host product before any production
// kernel relies on them.
#include <cuda_runtime.h>

#include <cstdint>

#include "umma.cuh"

namespace lio {
namespace {

__global__ void __launch_bounds__(128) k_tc_selftest(const int8_t* __restrict__ A, const int8_t* __restrict__ B,
                                                     int N, int K, int32_t* __restrict__ D, int* __restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  constexpr int M = 128;
  uint8_t* sA = smem;
  uint8_t* sB = smem + M * K;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t ncols = 32;
  while (ncols < (uint32_t)N) ncols <<= 1;
  if (warp == 0) umma::tmem_alloc(&tmem_base, ncols);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  for (int i = tid; i < M * K; i += blockDim.x) {
    const int r = i / K, k = i % K;
    sA[umma::kmajor_offset(r, k, M)] = (uint8_t)A[i];
  }
  for (int i = tid; i < N * K; i += blockDim.x) {
    const int r = i / K, k = i % K;
    sB[umma::kmajor_offset(r, k, N)] = (uint8_t)B[i];
  }
  umma::fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    const uint32_t idesc = umma::idesc_i8(M, N);
    const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
    for (int kk = 0; kk < K / 32; kk++) {
      const uint64_t ad = umma::smem_desc(a0 + 32u * M * kk, 16u * M, 128u);
      const uint64_t bd = umma::smem_desc(b0 + 32u * N * kk, 16u * N, 128u);
      umma::mma_i8(tbase, ad, bd, idesc, kk > 0 ? 1u : 0u);
    }
    umma::commit(&mbar);
  }
  const bool ok = umma::mbar_wait(&mbar, 0);
  umma::fence_after_sync();
  if (ok) {
    const int row = warp * 32 + lane;
    for (int c = 0; c < N; c += 8) {
      int32_t v[8];
      umma::tmem_ld8(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      umma::tmem_wait_ld();
      for (int j = 0; j < 8; j++) D[row * N + c + j] = v[j];
    }
  } else if (lane == 0) {
    atomicExch(status, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, ncols);
}

}  // namespace
}  // namespace lio

extern "C" __attribute__((visibility("default"))) int lio_tc_selftest_(int N, int K, const int8_t* hA,
                                                                       const int8_t* hB, int32_t* hD) {
  if (N < 16 || N > 256 || N % 16 || K < 32 || K % 32 || K > 256) return -2;
  int8_t *dA = nullptr, *dB = nullptr;
  int32_t* dD = nullptr;
  int* dS = nullptr;
  int status = -1;
  const size_t smem = (size_t)(128 + N) * K;
  if (cudaMalloc(&dA, 128 * K) != cudaSuccess || cudaMalloc(&dB, (size_t)N * K) != cudaSuccess ||
      cudaMalloc(&dD, (size_t)128 * N * 4) != cudaSuccess || cudaMalloc(&dS, sizeof(int)) != cudaSuccess)
    goto done;
  cudaMemcpy(dA, hA, 128 * K, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, hB, (size_t)N * K, cudaMemcpyHostToDevice);
  cudaMemset(dS, 0, sizeof(int));
  cudaMemset(dD, 0, (size_t)128 * N * 4);
  cudaFuncSetAttribute(lio::k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  lio::k_tc_selftest<<<1, 128, smem>>>(dA, dB, N, K, dD, dS);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    status = -3;
    goto done;
  }
  cudaMemcpy(&status, dS, sizeof(int), cudaMemcpyDeviceToHost);
  cudaMemcpy(hD, dD, (size_t)128 * N * 4, cudaMemcpyDeviceToHost);
done:
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(dS);
  return status;
}
