// Solver-level declarations (solver.cu, precond.cu, brownian.cu, integrator.cu).
#pragma once

#include "fsd_internal.h"

namespace fsd {

constexpr int kMaxRestart = 400;
constexpr int kMaxInner = 16;    // inner GMRES steps of the learned preconditioner
constexpr int kMaxPoly = 16;     // coefficients of the learned inner polynomial
constexpr int kPrunedCap = 32;   // pruned (r < rp) neighbours per particle, self included
constexpr int kSpaiCap = 32;     // members of a two-hop approximate-inverse set

// Leading dimension of the Krylov bases V and Z: 17N rounded up to 32 floats,
// so that every basis vector starts on a 128-byte boundary.
inline size_t krylov_ld(int N) { return (17 * (size_t)N + 31) & ~(size_t)31; }

int saddle_multiply(fsd_handle* h, const float4* pos, const float* x, float* b, bool rebin);
int precond_apply(fsd_handle* h, const float* b, float* x);
int saddle_solve(fsd_handle* h, const float4* pos, const float* b, float* x, float tol, int* iters, float* resid);
int gmres_alloc(fsd_handle* h);

// precond.cu: G ~ (R_FU^pruned + relaxer D)^-1 on 6N vectors.
int precond_alloc(fsd_handle* h);
void precond_free(fsd_handle* h);
int precond_build(fsd_handle* h, const float4* pos);
int precond_G(fsd_handle* h, const float* t, float* y);
int precond_apply_ichol(fsd_handle* h, const float* b, float* x);
int precond_wait_status(fsd_handle* h);
// Pruned R_FU + relaxer D in pruned-list order (precond.cu): pn (N), plist and
// blocks (N x kPrunedCap, self included), no ordering or factorisation.
int precond_assemble_pruned(fsd_handle* h, const float4* pos, float relaxer, const unsigned** pn,
                            const unsigned** plist, const float** blocks);

// Host reverse Cuthill-McKee ordering of a symmetric graph in CSR form
// (adjacency may include self loops).  perm[new] = old.
void rcm_order(int n, const std::vector<int>& rowptr, const std::vector<int>& col, std::vector<int>& perm);

}  // namespace fsd
