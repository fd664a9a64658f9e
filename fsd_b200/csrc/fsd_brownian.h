// Brownian and integrator declarations (brownian.cu, integrator.cu).
#pragma once

#include <functional>

#include "fsd_internal.h"

namespace fsd {

// Random streams of one time step (independent Philox key spaces).
constexpr uint32_t kStreamFFReal = 1;  // real-space far-field normals (11N)
constexpr uint32_t kStreamFFWave = 2;  // wave-space random field
constexpr uint32_t kStreamNF = 3;      // near-field normals (6N)
constexpr uint32_t kStreamRFD = 4;     // drift direction (6N)
constexpr uint32_t kStreamRot = 5;     // rotational noise (3N)
constexpr uint32_t kStreamGain = 6;    // start vector of the IC(0) gain estimate (6N)
constexpr uint32_t kStreamLearned = 7; // probe vectors of the learned preconditioner's training loss

void dot_device(fsd_handle* h, const float* a, const float* b, size_t n, double* out);
void gaussian(fsd_handle* h, float* out, size_t n, uint32_t step, uint32_t stream, float scale);
int lanczos_sqrt(fsd_handle* h, size_t n, const float* x, float* y, int* m_io, float tol, float scale,
                 const std::function<int(const float*, float*)>& apply, int* iters, float* err_out);
int brownian_farfield(fsd_handle* h, const float4* pos, uint32_t step, float* out11);
int brownian_nearfield(fsd_handle* h, const float4* pos, uint32_t step, float* out6);
int rfd_drift(fsd_handle* h, const float4* pos, uint32_t step, float* drift6);
bool tridiag_eigen(int m, std::vector<double>& d, std::vector<double> e, std::vector<double>& Z);

}  // namespace fsd
