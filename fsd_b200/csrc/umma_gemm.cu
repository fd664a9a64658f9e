// Tensor-core dense layers (placeholder until the tcgen05 kernels land).
#include "fsd_umma.h"

namespace fsd {

bool umma_gemm_supported(int, int) { return false; }
void umma_gemm(const float* const*, const int* const*, int, int, int, const float*, int, const float*, int,
               const float*, float*, cudaStream_t) {}
bool umma_gemm_dx_supported(int, int) { return false; }
void umma_gemm_dx(const float*, int, int, const float*, int, float*, cudaStream_t) {}

}  // namespace fsd
