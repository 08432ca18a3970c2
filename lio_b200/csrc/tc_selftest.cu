// Self-test of the tcgen05 int8 GEMM primitive (umma.cuh): D[128 x N] =
// A[128 x K] * B[N x K]^T with exact int32 accumulation in TMEM. Exposed as a
// C entry point so the GPU tests can check the descriptor encodings and the
// TMEM read-back layout against an exact host product before any production
// kernel relies on them.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

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

// The failure path of the pipelined kernels, exercised on purpose: a producer
// that stops early. It arms stage 0 of a two-stage ring and sends that stage's
// bulk copy, then stops without ever arming stage 1. The consumer waits for
// both stages with the caller's poll limit: stage 0 lands, stage 1's wait runs
// out. The consumer then does what the production kernels do after a timeout
// (records the failure, lets every copy it issued land, frees its TMEM) and
// the kernel returns, leaving the context usable. status: 0 both stages
// arrived, 1 a wait ran out, 2 stage 0 itself did not arrive.
__global__ void __launch_bounds__(64) k_wait_selftest(const uint4* __restrict__ src, uint32_t polls,
                                                      int* __restrict__ status, uint32_t* __restrict__ checksum) {
  __shared__ __align__(128) uint4 ring[2][64];  // two 1 KB stages
  __shared__ uint64_t full[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 32);
  if (tid == 0) {
    umma::mbar_init(&full[0], 1);
    umma::mbar_init(&full[1], 1);
    umma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 32) {  // producer: stage 0 only
    umma::mbar_expect_tx(&full[0], (uint32_t)sizeof(ring[0]));
    umma::bulk_copy_g2s(ring[0], src, (uint32_t)sizeof(ring[0]), &full[0]);
  }
  if (tid == 0) {  // consumer
    int st = 0;
    if (!umma::mbar_wait(&full[0], 0, polls)) {
      st = 2;
    } else {
      uint32_t sum = 0;
      for (int i = 0; i < 64; i++) sum += ring[0][i].x + ring[0][i].y + ring[0][i].z + ring[0][i].w;
      *checksum = sum;
      if (!umma::mbar_wait(&full[1], 0, polls)) st = 1;  // never armed: runs out
    }
    // the one copy issued lands before the CTA exits (the production limit,
    // not the caller's: a 1 KB copy takes microseconds)
    if (st == 2) umma::mbar_wait(&full[0], 0);
    *status = st;
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, 32);
}

}  // namespace

// Runs k_wait_selftest (one CTA) and returns its status; `ms` gets the
// kernel's device time (CUDA events). Throws on a CUDA error.
int bounded_wait_selftest(unsigned polls, double* ms, unsigned* checksum) {
  uint4* src = nullptr;
  int* dst = nullptr;
  int status = -1;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaMalloc(&src, 64 * sizeof(uint4));
  if (e == cudaSuccess) e = cudaMalloc(&dst, 2 * sizeof(int));
  if (e == cudaSuccess) {
    uint4 h[64];
    for (int i = 0; i < 64; i++) h[i] = make_uint4(4 * i, 4 * i + 1, 4 * i + 2, 4 * i + 3);
    e = cudaMemcpy(src, h, sizeof(h), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemset(dst, 0xff, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  if (e == cudaSuccess) {
    cudaEventRecord(a);
    k_wait_selftest<<<1, 64>>>(src, polls, dst, reinterpret_cast<uint32_t*>(dst + 1));
    e = cudaGetLastError();
    cudaEventRecord(b);
  }
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  int h[2] = {-1, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, dst, sizeof(h), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) {
    float f = 0.f;
    cudaEventElapsedTime(&f, a, b);
    if (ms) *ms = f;
    if (checksum) *checksum = (unsigned)h[1];
    status = h[0];
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(src);
  cudaFree(dst);
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in the bounded-wait self-test: ") +
                                                 cudaGetErrorString(e));
  return status;
}

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
