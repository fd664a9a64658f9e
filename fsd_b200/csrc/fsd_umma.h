// Dense layers of the message-passing network on the 5th-generation tensor
// cores (umma_gemm.cu): BF16 operands staged in shared memory, FP32
// accumulators in tensor memory.
#pragma once

#include <cuda_runtime.h>

namespace fsd {

// Y[r][o] = act(sum_k X(r, k) W[o][k] + b[o]) (+ resid[r][o]); X(r, :) is the
// concatenation of `parts` row-gathered pieces of `width` columns each.
bool umma_gemm_supported(int K, int O);
void umma_gemm(const float* const* p, const int* const* idx, int width, int parts, int rows, const float* Wt, int O,
               const float* bias, int relu, const float* resid, float* Y, cudaStream_t st);
// dX[r][k] = sum_o dY[r][o] W[o][k]
bool umma_gemm_dx_supported(int O, int K);
void umma_gemm_dx(const float* dY, int rows, int O, const float* Wt, int K, float* dX, cudaStream_t st);
// dW[o][k] += sum_r dY[r][o] X(r, k) and db[o] += sum_r dY[r][o]; `part`
// holds umma_dw_part_floats(rows, K, O) floats of per-CTA partial sums.
bool umma_gemm_dw_supported(int K, int O);
size_t umma_dw_part_floats(int rows, int K, int O);
void umma_gemm_dw(const float* const* p, const int* const* idx, int width, int parts, int rows, const float* dY,
                  int O, float* dW, float* db, float* part, cudaStream_t st);
// 1 if an mbarrier wait of these kernels ran out since the last call (then cleared); synchronises the device.
int umma_error();

}  // namespace fsd
