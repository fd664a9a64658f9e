// Near-field block preconditioner G ~ (R_FU^pruned + relaxer D)^-1
// (Precondition.cu / Helper_Precondition.cu of the reference).
//
//  1. pruned graph: each particle with itself and its neighbours closer than
//     rp = 2.1, sorted by index (Precondition_GetPrunedNlist_kernel);
//  2. R_FU restricted to that graph as 6x6 blocks (Precondition_RFU_kernel),
//     with relaxer * {1,1,1,4/3,4/3,4/3} added to the diagonal
//     (Precondition_AddIdentity_kernel);
//  3. reverse Cuthill-McKee ordering of the particle graph on the host
//     (genrcm, rcm.cpp:1009, restated in rcm_order below);
//  4. incomplete Cholesky with zero fill.  The scalar IC(0) of the reference
//     on a pattern made of dense 6x6 blocks equals block IC(0), which is what
//     is computed here, with FP64 arithmetic and pivots.  A pivot block that
//     is not positive definite either gets a local diagonal shift (default) or,
//     as the reference does, doubles the global relaxer and refactors
//     (Precondition.cu:1457-1489);
//  5. forward / backward block triangular solves, scheduled by dependency
//     level (one launch per level).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fsd_brownian.h"
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_solver.h"
#include "fsd_profile.h"

namespace fsd {

struct IChol {
    int N = 0;
    // device
    unsigned* pn = nullptr;      // pruned count per particle (self included)
    unsigned* plist = nullptr;   // N x kPrunedCap, sorted
    int* p_over = nullptr;       // overflow flag
    float* blocks = nullptr;     // assembled blocks, original row order: N x kPrunedCap x 36
    int* perm = nullptr;         // perm[new] = old
    int* rowptr = nullptr;       // permuted block CSR (N+1)
    int* col = nullptr;          // permuted column (new index), sorted
    int* src = nullptr;          // block slot in `blocks` for each CSR entry
    int* diag = nullptr;         // CSR position of the diagonal per row
    int* tpos = nullptr;         // CSR position of the transposed entry
    float* L = nullptr;          // factor blocks (fp32), per CSR entry, row-major 6x6
    float* Linv = nullptr;       // inverse of the diagonal factor block per row
    int* fail = nullptr;         // factorisation failure flag
    int* lev_rows = nullptr;     // rows sorted by forward level
    int* blev_rows = nullptr;    // rows sorted by backward level
    float* ty = nullptr;         // permuted work vector (6N)
    float* tz = nullptr;
    unsigned* ready_f = nullptr; // per-row completion epoch, forward solve
    unsigned* ready_b = nullptr; // per-row completion epoch, backward solve
    unsigned* tickets = nullptr; // row tickets [forward, backward]
    int* wait_err = nullptr;     // set when a bounded wait gave up
    float* gv = nullptr;         // gain estimate: two 17N saddle vectors
    double* gnrm = nullptr;      // device squared norm of the last iterate
    unsigned epoch = 0;
    int nnzb_cap = 0;
    // host
    std::vector<int> lev_ptr, blev_ptr;
    std::vector<unsigned> h_pn, h_plist;
    int nnzb = 0;
    int* h_fail = nullptr;
    double* h_gnrm = nullptr;
};

// ------------------------------------------------------------ pruned graph
__global__ void k_prune(const float4* __restrict__ pos, int N, Box b, const unsigned* __restrict__ nneigh,
                        const unsigned* __restrict__ nlist, int stride, float rp2, unsigned* pn, unsigned* plist,
                        int* over) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 pi = pos[i];
    unsigned* row = plist + (size_t)i * kPrunedCap;
    unsigned cnt = 1;
    row[0] = i;
    const unsigned nn = nneigh[i];
    for (unsigned q = 0; q < nn; ++q) {
        const unsigned j = nlist[(size_t)i * stride + q];
        const float4 pj = pos[j];
        const float3 r = min_image_rn(make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z), b);
        if (dist2_rn(r) < rp2) {
            if (cnt < kPrunedCap) row[cnt] = j;
            ++cnt;
        }
    }
    if (cnt > kPrunedCap) {
        atomicMax(over, (int)cnt);
        cnt = kPrunedCap;
    }
    for (unsigned a = 1; a < cnt; ++a) {
        const unsigned key = row[a];
        int c = (int)a - 1;
        while (c >= 0 && row[c] > key) {
            row[c + 1] = row[c];
            --c;
        }
        row[c + 1] = key;
    }
    pn[i] = cnt;
}

// Assemble the 6x6 blocks of particle i's pruned row (Precondition.cu:530-836):
//   neighbour block  [[A12, B12], [B12, C12]],  B12 = YB12 eps(r)
//   self block       sum over pruned neighbours [[A11, -B11], [B11, C11]]
// with the table's first row for r <= 2 + 1e-4, then relaxer on the diagonal.
__global__ void k_assemble(const float4* __restrict__ pos, int N, Box b, const unsigned* __restrict__ pn,
                           const unsigned* __restrict__ plist, ResTable tab, float rp, float relaxer, float* blocks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 pi = pos[i];
    const unsigned cnt = pn[i];
    const unsigned* row = plist + (size_t)i * kPrunedCap;
    float self[36];
#pragma unroll
    for (int k = 0; k < 36; ++k) self[k] = 0.0f;
    int self_slot = 0;
    const float rp2 = rp * rp;
    for (unsigned s = 0; s < cnt; ++s) {
        const unsigned j = row[s];
        float* blk = blocks + ((size_t)i * kPrunedCap + s) * 36;
        if (j == (unsigned)i) {
            self_slot = s;
            continue;
        }
        const float4 pj = pos[j];
        const float3 R = min_image_rn(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), b);
        const float d2 = dist2_rn(R);
        float c[10];
        if (!(d2 < rp2)) {
#pragma unroll
            for (int k = 0; k < 36; ++k) blk[k] = 0.0f;
            continue;
        }
        const float dist = sqrtf(d2);
        if ((double)dist <= (2.0 + (double)kResMin)) {
#pragma unroll
            for (int k = 0; k < 10; ++k) c[k] = __ldg(tab.vals + k);
        } else {
            const float sv = (float)(((double)dist - 2.0) / (double)kResMin);
            const int ind = (int)(log10f(sv) / kResDr);
            const float dl = __ldg(tab.dist + ind), du = __ldg(tab.dist + ind + 1);
            const float fac = (dist - dl) / (du - dl);
#pragma unroll
            for (int k = 0; k < 10; ++k) {
                const float lo = __ldg(tab.vals + 22 * ind + k), hi = __ldg(tab.vals + 22 * (ind + 1) + k);
                c[k] = lo + (hi - lo) * fac;
            }
        }
        const float XA11 = c[0], XA12 = c[1], YA11 = c[2], YA12 = c[3], YB11 = c[4], YB12 = c[5];
        const float XC11 = c[6], XC12 = c[7], YC11 = c[8], YC12 = c[9];
        const float r[3] = {R.x / dist, R.y / dist, R.z / dist};
        const float epsr[3][3] = {{0.0f, r[2], -r[1]}, {-r[2], 0.0f, r[0]}, {r[1], -r[0], 0.0f}};
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
                const float rr = r[ii] * r[jj];
                const float Imrr = (ii == jj ? 1.0f : 0.0f) - rr;
                const float An = XA12 * rr + YA12 * Imrr, As = XA11 * rr + YA11 * Imrr;
                const float Bn = YB12 * epsr[ii][jj], Bs = YB11 * epsr[ii][jj];
                const float Cn = XC12 * rr + YC12 * Imrr, Cs = XC11 * rr + YC11 * Imrr;
                blk[ii * 6 + jj] = An;
                blk[ii * 6 + jj + 3] = Bn;
                blk[(ii + 3) * 6 + jj] = Bn;
                blk[(ii + 3) * 6 + jj + 3] = Cn;
                self[ii * 6 + jj] += As;
                self[ii * 6 + jj + 3] += -Bs;
                self[(ii + 3) * 6 + jj] += Bs;
                self[(ii + 3) * 6 + jj + 3] += Cs;
            }
        }
    }
    float* sb = blocks + ((size_t)i * kPrunedCap + self_slot) * 36;
#pragma unroll
    for (int k = 0; k < 36; ++k) sb[k] = self[k];
#pragma unroll
    for (int d = 0; d < 6; ++d) sb[d * 7] += relaxer * ((d < 3) ? 1.0f : 1.33333333f);
}

// ------------------------------------------------------------- factorisation
// Block row p of the permuted matrix, rows of one level at a time.
//   L_pq = (B_pq - sum_{k<q} L_pk L_qk^T) L_qq^-T   for q < p in the pattern
//   L_pp = chol(B_pp - sum_{k<p} L_pk L_pk^T)
// FP64 throughout; a non-positive or non-finite pivot sets *fail.
// Cholesky of a 6x6 pivot block.  A pivot must keep at least kPivotFloor of
// the assembled diagonal entry `ref` it came from; smaller (or non-positive)
// pivots mark the block as failed, since a nearly singular pivot would give
// the preconditioner an enormous gain that swamps the FP32 Krylov basis.
constexpr double kPivotFloor = 1e-3;
constexpr int kGainIters = 8;  // power-iteration steps of the gain estimate

__device__ void chol6(double* A, bool* ok, const float* ref) {
    for (int j = 0; j < 6; ++j) {
        double d = A[j * 6 + j];
        for (int k = 0; k < j; ++k) d -= A[j * 6 + k] * A[j * 6 + k];
        const double floor_j = ref ? kPivotFloor * fabs((double)ref[j * 7]) : 0.0;
        if (!(d > floor_j) || !(d > 0.0)) {
            *ok = false;
            d = 1.0;
        }
        d = sqrt(d);
        A[j * 6 + j] = d;
        for (int i = j + 1; i < 6; ++i) {
            double v = A[i * 6 + j];
            for (int k = 0; k < j; ++k) v -= A[i * 6 + k] * A[j * 6 + k];
            A[i * 6 + j] = v / d;
        }
        for (int k = j + 1; k < 6; ++k) A[j * 6 + k] = 0.0;
    }
}

__global__ void k_factor_level(const int* __restrict__ rows, int nrows, const int* __restrict__ rowptr,
                               const int* __restrict__ col, const int* __restrict__ src, const int* __restrict__ diag,
                               const float* __restrict__ blocks, float* L, float* Linv, int* fail, bool local_shift,
                               double shift0, int* shifted) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    const int p = rows[t];
    const int b = rowptr[p], dp = diag[p];
    double acc[36];
    for (int e = b; e <= dp; ++e) {
        const int q = col[e];
        const float* B = blocks + (size_t)src[e] * 36;
        for (int k = 0; k < 36; ++k) acc[k] = (double)B[k];
        // subtract sum_{k < q} L_pk L_qk^T over the common pattern
        const int bq = rowptr[q], dq = diag[q];
        int ip = b, iq = bq;
        while (ip < e && iq < dq) {
            const int cp = col[ip], cq = col[iq];
            if (cp == cq) {
                const float* Lp = L + (size_t)ip * 36;
                const float* Lq = L + (size_t)iq * 36;
                for (int r = 0; r < 6; ++r)
                    for (int c = 0; c < 6; ++c) {
                        double s = 0.0;
                        for (int k = 0; k < 6; ++k) s += (double)Lp[r * 6 + k] * (double)Lq[c * 6 + k];
                        acc[r * 6 + c] -= s;
                    }
                ++ip;
                ++iq;
            } else if (cp < cq) {
                ++ip;
            } else {
                ++iq;
            }
        }
        float* out = L + (size_t)e * 36;
        if (e < dp) {
            // acc <- acc * L_qq^-T : solve X L_qq^T = acc row by row
            const float* Lqq = L + (size_t)dq * 36;
            for (int r = 0; r < 6; ++r) {
                for (int c = 0; c < 6; ++c) {
                    double v = acc[r * 6 + c];
                    for (int k = 0; k < c; ++k) v -= acc[r * 6 + k] * (double)Lqq[c * 6 + k];
                    acc[r * 6 + c] = v / (double)Lqq[c * 6 + c];
                }
            }
            for (int k = 0; k < 36; ++k) out[k] = (float)acc[k];
        } else {
            bool ok = true;
            double keep[36];
            for (int k = 0; k < 36; ++k) keep[k] = acc[k];
            chol6(acc, &ok, B);
            // Pivot-local shift: a pivot block that is not positive definite
            // gets tau * {1,1,1,4/3,4/3,4/3} added, tau doubling from
            // `shift0`, instead of shifting the whole matrix.
            if (!ok && local_shift) {
                double tau = shift0;
                for (int attempt = 0; attempt < 40 && !ok; ++attempt, tau *= 2.0) {
                    for (int k = 0; k < 36; ++k) acc[k] = keep[k];
                    for (int d = 0; d < 6; ++d) acc[d * 7] += tau * ((d < 3) ? 1.0 : (double)1.33333333f);
                    ok = true;
                    chol6(acc, &ok, B);
                }
                if (ok) atomicAdd(shifted, 1);
            }
            if (!ok) atomicExch(fail, 1);
            for (int k = 0; k < 36; ++k) out[k] = (float)acc[k];
            // inverse of the lower-triangular factor, forward substitution on I
            double inv[36];
            for (int k = 0; k < 36; ++k) inv[k] = 0.0;
            for (int c = 0; c < 6; ++c) {
                for (int r = c; r < 6; ++r) {
                    double v = (r == c) ? 1.0 : 0.0;
                    for (int k = c; k < r; ++k) v -= acc[r * 6 + k] * inv[k * 6 + c];
                    inv[r * 6 + c] = v / acc[r * 6 + r];
                }
            }
            float* li = Linv + (size_t)p * 36;
            for (int k = 0; k < 36; ++k) li[k] = (float)inv[k];
        }
    }
}

// ---------------------------------------------------------------- solves
// Forward: z_p = Linv_pp (t_p - sum_{q<p} L_pq z_q), on permuted vectors.
__global__ void k_fwd_level(const int* __restrict__ rows, int nrows, const int* __restrict__ rowptr,
                            const int* __restrict__ col, const int* __restrict__ diag, const float* __restrict__ L,
                            const float* __restrict__ Linv, const float* __restrict__ t, float* z) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int p = rows[k];
    float v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = t[6 * p + c];
    for (int e = rowptr[p]; e < diag[p]; ++e) {
        const int q = col[e];
        const float* B = L + (size_t)e * 36;
        float zq[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) zq[c] = z[6 * q + c];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 6; ++c) s += B[r * 6 + c] * zq[c];
            v[r] -= s;
        }
    }
    const float* Li = Linv + (size_t)p * 36;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c <= r; ++c) s += Li[r * 6 + c] * v[c];
        z[6 * p + r] = s;
    }
}

// Backward: x_p = Linv_pp^T (z_p - sum_{q>p} L_qp^T x_q).
__global__ void k_bwd_level(const int* __restrict__ rows, int nrows, const int* __restrict__ rowptr,
                            const int* __restrict__ col, const int* __restrict__ diag, const int* __restrict__ tpos,
                            const float* __restrict__ L, const float* __restrict__ Linv, const float* __restrict__ z,
                            float* x) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int p = rows[k];
    float v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = z[6 * p + c];
    for (int e = diag[p] + 1; e < rowptr[p + 1]; ++e) {
        const int q = col[e];
        const float* B = L + (size_t)tpos[e] * 36;  // L_qp
        float xq[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) xq[c] = x[6 * q + c];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 6; ++c) s += B[c * 6 + r] * xq[c];
            v[r] -= s;
        }
    }
    const float* Li = Linv + (size_t)p * 36;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        float s = 0.0f;
#pragma unroll
        for (int c = r; c < 6; ++c) s += Li[c * 6 + r] * v[c];
        x[6 * p + r] = s;
    }
}

__global__ void k_permute(const float* __restrict__ in, float* __restrict__ out, const int* __restrict__ perm, int N,
                          int dir) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 6 * N) return;
    const int p = k / 6, c = k % 6;
    if (dir > 0)
        out[k] = in[6 * perm[p] + c];  // to permuted order
    else
        out[6 * perm[p] + c] = in[k];  // back to original order
}

// ------------------------------------------------------- sync-free solves
// One launch per triangular solve.  Warps take rows in dependency order from
// a ticket counter, so every row a warp waits on belongs to a warp that is
// already running; a finished row publishes its values, then its epoch flag.
// Each wait is bounded: after kWaitLimit polls the kernel records the row in
// *err and carries on, so a fault in the schedule cannot hang the GPU.
constexpr int kWaitLimit = 1 << 22;

__device__ __forceinline__ void wait_ready(const unsigned* flag, unsigned epoch, int* err, int row) {
    int n = 0;
    while (*(volatile const unsigned*)flag != epoch) {
        if (++n > kWaitLimit) {
            atomicExch(err, row + 1);
            break;
        }
        __nanosleep(32);
    }
    __threadfence();
}

// Forward solve with the saddle pre-step fused: for permuted row p with
// particle i = perm[p], t_p = b[6i:6i+6] - b[11N+6i:11N+6i+6], then
// z_p = Linv_pp (t_p - sum_{q<p} L_pq z_q).  Also copies b[6N:11N] to x.
__global__ void __launch_bounds__(128) k_trsv_fwd(const int* __restrict__ order, int N, const int* __restrict__ perm,
                                                  const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const int* __restrict__ diag, const float* __restrict__ L,
                                                  const float* __restrict__ Linv, const float* __restrict__ b,
                                                  float* __restrict__ x, float* z, unsigned* ready, unsigned epoch,
                                                  unsigned* ticket, int* err) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned tk = 0;
        if (lane == 0) tk = atomicAdd(ticket, 1u);
        tk = __shfl_sync(0xffffffffu, tk, 0);
        if (tk >= (unsigned)N) return;
        const int p = order[tk];
        const int i = perm[p];
        float v = 0.f;
        if (lane < 6) v = b[6 * i + lane] - b[11 * (size_t)N + 6 * i + lane];
        if (lane < 5) x[6 * (size_t)N + 5 * i + lane] = b[6 * (size_t)N + 5 * i + lane];
        for (int e = rowptr[p]; e < diag[p]; ++e) {
            const int q = col[e];
            if (lane == 0) wait_ready(ready + q, epoch, err, q);
            __syncwarp();
            float zq = (lane < 6) ? __ldcg(z + 6 * q + lane) : 0.f;
            const float* B = L + (size_t)e * 36;
            float acc = 0.f;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                const float zd = __shfl_sync(0xffffffffu, zq, d);
                if (lane < 6) acc += B[lane * 6 + d] * zd;
            }
            v -= acc;
        }
        const float* Li = Linv + (size_t)p * 36;
        float out = 0.f;
#pragma unroll
        for (int d = 0; d < 6; ++d) {
            const float vd = __shfl_sync(0xffffffffu, v, d);
            if (lane < 6 && d <= lane) out += Li[lane * 6 + d] * vd;
        }
        if (lane < 6) __stcg(z + 6 * p + lane, out);
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicExch(ready + p, epoch);
    }
}

// Backward solve with the saddle post-step fused: x_p = Linv_pp^T (z_p -
// sum_{q>p} L_qp^T x_q); particle i = perm[p] gets y = x_p:
// out[6i:6i+6] = b[6i:6i+6] - y and out[11N+6i:11N+6i+6] = y.
__global__ void __launch_bounds__(128) k_trsv_bwd(const int* __restrict__ order, int N, const int* __restrict__ perm,
                                                  const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const int* __restrict__ diag, const int* __restrict__ tpos,
                                                  const float* __restrict__ L, const float* __restrict__ Linv,
                                                  const float* __restrict__ z, const float* __restrict__ b,
                                                  float* __restrict__ out, float* xp, unsigned* ready, unsigned epoch,
                                                  unsigned* ticket, int* err) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned tk = 0;
        if (lane == 0) tk = atomicAdd(ticket, 1u);
        tk = __shfl_sync(0xffffffffu, tk, 0);
        if (tk >= (unsigned)N) return;
        const int p = order[tk];
        float v = (lane < 6) ? __ldcg(z + 6 * p + lane) : 0.f;
        for (int e = diag[p] + 1; e < rowptr[p + 1]; ++e) {
            const int q = col[e];
            if (lane == 0) wait_ready(ready + q, epoch, err, q);
            __syncwarp();
            float xq = (lane < 6) ? __ldcg(xp + 6 * q + lane) : 0.f;
            const float* B = L + (size_t)tpos[e] * 36;  // L_qp
            float acc = 0.f;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const float xc = __shfl_sync(0xffffffffu, xq, c);
                if (lane < 6) acc += B[c * 6 + lane] * xc;
            }
            v -= acc;
        }
        const float* Li = Linv + (size_t)p * 36;
        float y = 0.f;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float vc = __shfl_sync(0xffffffffu, v, c);
            if (lane < 6 && c >= lane) y += Li[c * 6 + lane] * vc;
        }
        if (lane < 6) {
            __stcg(xp + 6 * p + lane, y);
            const int i = perm[p];
            out[6 * i + lane] = b[6 * i + lane] - y;
            out[11 * (size_t)N + 6 * i + lane] = y;
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicExch(ready + p, epoch);
    }
}

// -------------------------------------------------------------- host RCM
namespace {
// Breadth-first level structure from root over unmasked nodes; returns the
// number of levels, nodes in `order`, level starts in `lstart`.
int level_structure(int root, const std::vector<int>& rp, const std::vector<int>& cl, std::vector<char>& mask,
                    std::vector<int>& order, std::vector<int>& lstart) {
    order.clear();
    lstart.clear();
    order.push_back(root);
    mask[root] = 0;
    size_t lb = 0;
    int nl = 0;
    for (;;) {
        const size_t le = order.size();
        lstart.push_back((int)lb);
        ++nl;
        for (size_t i = lb; i < le; ++i) {
            const int v = order[i];
            for (int e = rp[v]; e < rp[v + 1]; ++e) {
                const int u = cl[e];
                if (mask[u]) {
                    mask[u] = 0;
                    order.push_back(u);
                }
            }
        }
        if (order.size() == le) break;
        lb = le;
    }
    lstart.push_back((int)order.size());
    for (int v : order) mask[v] = 1;
    return nl;
}
}  // namespace

void rcm_order(int n, const std::vector<int>& rp, const std::vector<int>& cl, std::vector<int>& perm) {
    std::vector<char> mask(n, 1);
    std::vector<int> order, lstart, deg(n, 0);
    perm.clear();
    perm.reserve(n);
    for (int start = 0; start < n; ++start) {
        if (!mask[start]) continue;
        // Pseudo-peripheral root (George & Liu).
        int root = start;
        int nl = level_structure(root, rp, cl, mask, order, lstart);
        const int csize = (int)order.size();
        if (nl > 1 && nl != csize) {
            for (;;) {
                int mindeg = csize;
                const int ls = lstart[nl - 1];
                root = order[ls];
                for (int k = ls; k < csize; ++k) {
                    const int v = order[k];
                    int d = 0;
                    for (int e = rp[v]; e < rp[v + 1]; ++e) d += mask[cl[e]] > 0;
                    if (d < mindeg) {
                        root = v;
                        mindeg = d;
                    }
                }
                std::vector<int> o2, l2;
                const int nl2 = level_structure(root, rp, cl, mask, o2, l2);
                if (nl2 <= nl) break;
                nl = nl2;
                order.swap(o2);
                lstart.swap(l2);
                if (csize <= nl) break;
            }
        }
        // Degrees within the component (unmasked neighbours, self loops counted).
        level_structure(root, rp, cl, mask, order, lstart);
        for (int v : order) {
            int d = 0;
            for (int e = rp[v]; e < rp[v + 1]; ++e) d += mask[cl[e]] != 0;
            deg[v] = d;
        }
        // Cuthill-McKee: breadth first, each node's new neighbours by increasing degree.
        const size_t base = perm.size();
        perm.push_back(root);
        mask[root] = 0;
        size_t lvlend = base, lnbr = base + 1;
        while (lvlend < lnbr) {
            const size_t lbegin = lvlend;
            lvlend = lnbr;
            for (size_t i = lbegin; i < lvlend; ++i) {
                const int v = perm[i];
                const size_t fnbr = perm.size();
                for (int e = rp[v]; e < rp[v + 1]; ++e) {
                    const int u = cl[e];
                    if (mask[u]) {
                        mask[u] = 0;
                        perm.push_back(u);
                    }
                }
                // Stable insertion sort by degree of the new neighbours after
                // the first one; the first stays in place, as in the
                // reference's genrcm (rcm.cpp, inner loop `while ( fnbr < l )`).
                for (size_t k = fnbr + 2; k < perm.size(); ++k) {
                    const int key = perm[k];
                    size_t l = k;
                    while (l > fnbr + 1 && deg[perm[l - 1]] > deg[key]) {
                        perm[l] = perm[l - 1];
                        --l;
                    }
                    perm[l] = key;
                }
                lnbr = perm.size();
            }
        }
        std::reverse(perm.begin() + base, perm.end());
    }
}

// ------------------------------------------------------------ host driver
int precond_alloc(fsd_handle* h) {
    IChol* ic = new IChol();
    h->ichol = ic;
    const int N = h->p.N;
    ic->N = N;
    ic->nnzb_cap = N * kPrunedCap;
    FSD_CHECK_CUDA(cudaMalloc(&ic->pn, sizeof(unsigned) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->plist, sizeof(unsigned) * (size_t)N * kPrunedCap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->p_over, sizeof(int)));
    FSD_CHECK_CUDA(cudaMalloc(&ic->blocks, sizeof(float) * 36 * (size_t)N * kPrunedCap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->perm, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->rowptr, sizeof(int) * (N + 1)));
    FSD_CHECK_CUDA(cudaMalloc(&ic->col, sizeof(int) * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->src, sizeof(int) * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->diag, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->tpos, sizeof(int) * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->L, sizeof(float) * 36 * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->Linv, sizeof(float) * 36 * (size_t)N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->fail, sizeof(int) * 2));
    FSD_CHECK_CUDA(cudaMalloc(&ic->lev_rows, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->blev_rows, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->ty, sizeof(float) * 6 * (size_t)N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->tz, sizeof(float) * 6 * (size_t)N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->ready_f, sizeof(unsigned) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->ready_b, sizeof(unsigned) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->tickets, sizeof(unsigned) * 2));
    FSD_CHECK_CUDA(cudaMalloc(&ic->wait_err, sizeof(int)));
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->ready_f, 0, sizeof(unsigned) * N, h->stream));
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->ready_b, 0, sizeof(unsigned) * N, h->stream));
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->wait_err, 0, sizeof(int), h->stream));
    FSD_CHECK_CUDA(cudaMalloc(&ic->gv, sizeof(float) * 34 * (size_t)N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->gnrm, sizeof(double)));
    FSD_CHECK_CUDA(cudaMallocHost(&ic->h_fail, sizeof(int) * 2));
    FSD_CHECK_CUDA(cudaMallocHost(&ic->h_gnrm, sizeof(double)));
    return FSD_OK;
}

void precond_free(fsd_handle* h) {
    IChol* ic = (IChol*)h->ichol;
    if (!ic) return;
    void* ptrs[] = {ic->pn, ic->plist, ic->p_over, ic->blocks, ic->perm, ic->rowptr, ic->col, ic->src, ic->diag,
                    ic->tpos, ic->L, ic->Linv, ic->fail, ic->lev_rows, ic->blev_rows, ic->ty, ic->tz,
                    ic->ready_f, ic->ready_b, ic->tickets, ic->wait_err, ic->gv, ic->gnrm};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (ic->h_fail) cudaFreeHost(ic->h_fail);
    if (ic->h_gnrm) cudaFreeHost(ic->h_gnrm);
    delete ic;
    h->ichol = nullptr;
}

// y = x / sqrt(*nrm) (a zero norm leaves y = x).
__global__ void k_normalize(float* __restrict__ y, const float* __restrict__ x, const double* __restrict__ nrm,
                            size_t n) {
    const double s = *nrm;
    const float f = s > 0.0 ? (float)(1.0 / sqrt(s)) : 1.0f;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        y[k] = f * x[k];
}

// Power-iteration estimate of lambda_max(G) for the current factor.  With the
// saddle input b = [0; u] the preconditioner returns G u in its last 6N
// entries, so the iteration runs on the fused solve kernels unchanged.
// The iteration count is small: a factor that has lost stability has a gain
// many orders of magnitude above 1/relaxer, which a few steps expose.
double ichol_gain(fsd_handle* h, int iters) {
    IChol* ic = (IChol*)h->ichol;
    const int N = h->p.N;
    const size_t n6 = 6 * (size_t)N, off = 11 * (size_t)N;
    cudaStream_t st = h->stream;
    float* b = ic->gv;
    float* x = ic->gv + 17 * (size_t)N;
    const int nb = (int)std::min<size_t>(4 * 148, (n6 + 255) / 256);
    if (cudaMemsetAsync(b, 0, sizeof(float) * off, st) != cudaSuccess) return -1.0;
    gaussian(h, b + off, n6, 0, kStreamGain, 1.0f);
    dot_device(h, b + off, b + off, n6, ic->gnrm);
    count_launch();
    k_normalize<<<nb, 256, 0, st>>>(b + off, b + off, ic->gnrm, n6);
    for (int it = 0; it < iters; ++it) {
        if (precond_apply_ichol(h, b, x) != FSD_OK) return -1.0;
        dot_device(h, x + off, x + off, n6, ic->gnrm);
        count_launch();
        k_normalize<<<nb, 256, 0, st>>>(b + off, x + off, ic->gnrm, n6);
    }
    if (cudaMemcpyAsync(ic->h_gnrm, ic->gnrm, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1.0;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1.0;
    return sqrt(*ic->h_gnrm);
}

// Build the pattern, ordering and levels from the pruned graph (host), then
// factor with the current relaxer, doubling it on failure.
int precond_build(fsd_handle* h, const float4* pos) {
    IChol* ic = (IChol*)h->ichol;
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    if (h->p.precond == FSD_PRECOND_NONE) {
        h->pc_valid = true;
        return FSD_OK;
    }
    if (h->p.precond == FSD_PRECOND_LEARNED) return precond_build_learned(h, pos);
    ProfRegion pr(h, R_PRECOND_BUILD);
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->p_over, 0, sizeof(int), st));
    count_launch();
    k_prune<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, h->w.nneigh, h->w.nlist, h->w.nl_stride,
                                             h->p.rp * h->p.rp, ic->pn, ic->plist, ic->p_over);
    ic->h_pn.resize(N);
    ic->h_plist.resize((size_t)N * kPrunedCap);
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_pn.data(), ic->pn, sizeof(unsigned) * N, cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_plist.data(), ic->plist, sizeof(unsigned) * (size_t)N * kPrunedCap,
                                   cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_fail, ic->p_over, sizeof(int), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    if (ic->h_fail[0] > 0) return FSD_ERR_NLIST_OVERFLOW;
    // Particle graph in CSR (self loops included, rows sorted).
    std::vector<int> rp(N + 1, 0), cl;
    cl.reserve((size_t)N * 6);
    for (int i = 0; i < N; ++i) {
        for (unsigned s = 0; s < ic->h_pn[i]; ++s) cl.push_back((int)ic->h_plist[(size_t)i * kPrunedCap + s]);
        rp[i + 1] = (int)cl.size();
    }
    std::vector<int> perm, inv(N);
    rcm_order(N, rp, cl, perm);
    for (int p = 0; p < N; ++p) inv[perm[p]] = p;
    // Permuted block CSR with sorted new-index columns.
    std::vector<int> prow(N + 1, 0), pcol, psrc, pdiag(N), ptpos;
    pcol.reserve(cl.size());
    psrc.reserve(cl.size());
    std::vector<std::pair<int, int>> tmp;
    for (int p = 0; p < N; ++p) {
        const int i = perm[p];
        tmp.clear();
        for (int e = rp[i]; e < rp[i + 1]; ++e) tmp.emplace_back(inv[cl[e]], i * kPrunedCap + (e - rp[i]));
        std::sort(tmp.begin(), tmp.end());
        for (auto& t : tmp) {
            if (t.first == p) pdiag[p] = (int)pcol.size();
            pcol.push_back(t.first);
            psrc.push_back(t.second);
        }
        prow[p + 1] = (int)pcol.size();
    }
    const int nnzb = (int)pcol.size();
    ic->nnzb = nnzb;
    ptpos.assign(nnzb, -1);
    for (int p = 0; p < N; ++p)
        for (int e = prow[p]; e < prow[p + 1]; ++e) {
            const int q = pcol[e];
            // position of (q, p) in row q (pattern is symmetric)
            const int* b = pcol.data() + prow[q];
            const int* en = pcol.data() + prow[q + 1];
            const int* f = std::lower_bound(b, en, p);
            ptpos[e] = (f != en && *f == p) ? (int)(f - pcol.data()) : -1;
        }
    // Dependency levels (forward and backward).
    std::vector<int> lev(N, 0), blev(N, 0);
    int nlev = 0, nblev = 0;
    for (int p = 0; p < N; ++p) {
        int l = 0;
        for (int e = prow[p]; e < pdiag[p]; ++e) l = std::max(l, lev[pcol[e]] + 1);
        lev[p] = l;
        nlev = std::max(nlev, l + 1);
    }
    for (int p = N - 1; p >= 0; --p) {
        int l = 0;
        for (int e = pdiag[p] + 1; e < prow[p + 1]; ++e) l = std::max(l, blev[pcol[e]] + 1);
        blev[p] = l;
        nblev = std::max(nblev, l + 1);
    }
    auto bucket = [N](const std::vector<int>& lv, int nl, std::vector<int>& ptr, std::vector<int>& rows) {
        ptr.assign(nl + 1, 0);
        for (int p = 0; p < N; ++p) ptr[lv[p] + 1]++;
        for (int l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
        rows.resize(N);
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int p = 0; p < N; ++p) rows[fill[lv[p]]++] = p;
    };
    std::vector<int> lrows, brows;
    bucket(lev, nlev, ic->lev_ptr, lrows);
    bucket(blev, nblev, ic->blev_ptr, brows);
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->perm, perm.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->rowptr, prow.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->col, pcol.data(), sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->src, psrc.data(), sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->diag, pdiag.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->tpos, ptpos.data(), sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->lev_rows, lrows.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->blev_rows, brows.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    h->info.ichol_attempts = 0;
    // Factor, doubling the relaxer after each failure (Precondition.cu:1457-1489).
    for (int attempt = 0; attempt < 24; ++attempt) {
        count_launch();
        k_assemble<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, ic->pn, ic->plist,
                                                   ResTable{h->d_res_dist, h->d_res_vals}, h->p.rp, h->ichol_relaxer,
                                                   ic->blocks);
        FSD_CHECK_CUDA(cudaMemsetAsync(ic->fail, 0, sizeof(int) * 2, st));
        for (int l = 0; l < nlev; ++l) {
            const int n = ic->lev_ptr[l + 1] - ic->lev_ptr[l];
            count_launch();
            k_factor_level<<<(n + 63) / 64, 64, 0, st>>>(ic->lev_rows + ic->lev_ptr[l], n, ic->rowptr, ic->col,
                                                        ic->src, ic->diag, ic->blocks, ic->L, ic->Linv, ic->fail,
                                                        h->p.ichol_local_shift != 0, (double)h->ichol_relaxer,
                                                        ic->fail + 1);
        }
        FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_fail, ic->fail, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
        FSD_CHECK_CUDA(cudaStreamSynchronize(st));
        h->info.ichol_attempts = attempt + 1;
        h->info.ichol_shifted = ic->h_fail[1];
        if (!ic->h_fail[0]) {
            // Stability check: IC(0) of the pruned lubrication matrix can be
            // positive definite yet nearly singular (dropped fill around
            // clusters of touching spheres); its inverse then amplifies some
            // directions by many orders of magnitude and GMRES stagnates.
            double gain = 0.0;
            if (h->p.ichol_gain_limit > 0.f) {
                gain = ichol_gain(h, kGainIters);
                if (gain < 0.0) return FSD_ERR_CUDA;
                const int ws = precond_wait_status(h);
                if (ws != FSD_OK) return ws;
            }
            h->info.ichol_gain = (float)gain;
            if (h->p.ichol_gain_limit <= 0.f || gain * h->ichol_relaxer <= h->p.ichol_gain_limit) {
                h->info.ichol_relaxer = h->ichol_relaxer;
                h->pc_valid = true;
                return FSD_OK;
            }
        }
        h->ichol_relaxer *= 2.0f;
    }
    return FSD_ERR_ICHOL;
}

// Pruned matrix only (for preconditioners that use R_FU^pruned + relaxer D as
// an operator): prune, check the list capacity, assemble.
int precond_assemble_pruned(fsd_handle* h, const float4* pos, float relaxer, const unsigned** pn,
                            const unsigned** plist, const float** blocks) {
    IChol* ic = (IChol*)h->ichol;
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->p_over, 0, sizeof(int), st));
    count_launch();
    k_prune<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, h->w.nneigh, h->w.nlist, h->w.nl_stride,
                                             h->p.rp * h->p.rp, ic->pn, ic->plist, ic->p_over);
    count_launch();
    k_assemble<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, ic->pn, ic->plist,
                                               ResTable{h->d_res_dist, h->d_res_vals}, h->p.rp, relaxer, ic->blocks);
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_fail, ic->p_over, sizeof(int), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    if (ic->h_fail[0] > 0) return FSD_ERR_NLIST_OVERFLOW;
    *pn = ic->pn;
    *plist = ic->plist;
    *blocks = ic->blocks;
    return FSD_OK;
}

// x = P^-1 b for the saddle system with the IC(0) factor, two launches.
int precond_apply_ichol(fsd_handle* h, const float* b, float* x) {
    IChol* ic = (IChol*)h->ichol;
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    ic->epoch += 1;
    if (ic->epoch == 0) {  // wrapped: clear the flags once
        FSD_CHECK_CUDA(cudaMemsetAsync(ic->ready_f, 0, sizeof(unsigned) * N, st));
        FSD_CHECK_CUDA(cudaMemsetAsync(ic->ready_b, 0, sizeof(unsigned) * N, st));
        ic->epoch = 1;
    }
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->tickets, 0, sizeof(unsigned) * 2, st));
    const int warps = std::min(N, 148 * 16);
    const int blocks = (warps * 32 + 127) / 128;
    count_launch();
    k_trsv_fwd<<<blocks, 128, 0, st>>>(ic->lev_rows, N, ic->perm, ic->rowptr, ic->col, ic->diag, ic->L, ic->Linv, b, x,
                                       ic->tz, ic->ready_f, ic->epoch, ic->tickets, ic->wait_err);
    count_launch();
    k_trsv_bwd<<<blocks, 128, 0, st>>>(ic->blev_rows, N, ic->perm, ic->rowptr, ic->col, ic->diag, ic->tpos, ic->L,
                                       ic->Linv, ic->tz, b, x, ic->ty, ic->ready_b, ic->epoch, ic->tickets + 1,
                                       ic->wait_err);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Bounded-wait failures since the last call (0 = none); clears the flag.
int precond_wait_status(fsd_handle* h) {
    IChol* ic = (IChol*)h->ichol;
    if (!ic || !ic->wait_err) return FSD_OK;
    int v = 0;
    FSD_CHECK_CUDA(cudaMemcpyAsync(&v, ic->wait_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (v) {
        FSD_CHECK_CUDA(cudaMemsetAsync(ic->wait_err, 0, sizeof(int), h->stream));
        return FSD_ERR_DEVICE_WAIT;
    }
    return FSD_OK;
}

int precond_G(fsd_handle* h, const float* t, float* y) {
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    if (h->p.precond == FSD_PRECOND_NONE) {
        FSD_CHECK_CUDA(cudaMemcpyAsync(y, t, sizeof(float) * 6 * N, cudaMemcpyDeviceToDevice, st));
        return FSD_OK;
    }
    IChol* ic = (IChol*)h->ichol;
    count_launch();
    k_permute<<<(6 * N + 255) / 256, 256, 0, st>>>(t, ic->ty, ic->perm, N, 1);
    const int nlev = (int)ic->lev_ptr.size() - 1;
    for (int l = 0; l < nlev; ++l) {
        const int n = ic->lev_ptr[l + 1] - ic->lev_ptr[l];
        count_launch();
        k_fwd_level<<<(n + 127) / 128, 128, 0, st>>>(ic->lev_rows + ic->lev_ptr[l], n, ic->rowptr, ic->col, ic->diag,
                                                     ic->L, ic->Linv, ic->ty, ic->tz);
    }
    const int nblev = (int)ic->blev_ptr.size() - 1;
    for (int l = 0; l < nblev; ++l) {
        const int n = ic->blev_ptr[l + 1] - ic->blev_ptr[l];
        count_launch();
        k_bwd_level<<<(n + 127) / 128, 128, 0, st>>>(ic->blev_rows + ic->blev_ptr[l], n, ic->rowptr, ic->col,
                                                     ic->diag, ic->tpos, ic->L, ic->Linv, ic->tz, ic->ty);
    }
    count_launch();
    k_permute<<<(6 * N + 255) / 256, 256, 0, st>>>(ic->ty, y, ic->perm, N, -1);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

}  // namespace fsd
