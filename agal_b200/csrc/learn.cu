// Learned refinement predictor: a small convolutional network over per-block
// fields that predicts the refine / coarsen marks of the next regrid, trained
// on the GPU on snapshots of the plain criterion (no reference counterpart;
// the reference only has the plain vorticity / Q criterion).
//
// This file: the tensor-core GEMM entry point used by the network's layers.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

#include "ctx.h"
#include "umma_gemm.cuh"

extern "C" int agal_learn_gemm_bf16(const uint16_t *A, const uint16_t *B, float *D, int M, int N, int K)
{
    // D[M x N] = A[M x K] . B[N x K]^T on host buffers (BF16 bit patterns in,
    // FP32 out) through the tcgen05 kernel; a test hook of the layers' GEMM.
    if (!A || !B || !D || M <= 0 || N < 1 || N > agal::umma::TN || K <= 0 || K % 16) return AGAL_ERR_PARAM;
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float *dD = nullptr;
    int *st = nullptr;
    int rc = AGAL_OK, hs = 0;
    if (cudaMalloc(&dA, sizeof(uint16_t) * (size_t)M * K) != cudaSuccess ||
        cudaMalloc(&dB, sizeof(uint16_t) * (size_t)N * K) != cudaSuccess ||
        cudaMalloc(&dD, sizeof(float) * (size_t)M * N) != cudaSuccess || cudaMalloc(&st, sizeof(int)) != cudaSuccess) {
        rc = AGAL_ERR_OOM;
    } else if (cudaMemcpy(dA, A, sizeof(uint16_t) * (size_t)M * K, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(dB, B, sizeof(uint16_t) * (size_t)N * K, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemset(st, 0, sizeof(int)) != cudaSuccess ||
               agal::umma::gemm_bf16(dA, dB, dD, M, N, K, N, st, 0) != cudaSuccess ||
               cudaDeviceSynchronize() != cudaSuccess ||
               cudaMemcpy(D, dD, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost) != cudaSuccess ||
               cudaMemcpy(&hs, st, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = AGAL_ERR_CUDA;
    } else if (hs) {
        rc = hs;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(st);
    return rc;
}
