// Saddle-point operator, its block preconditioner and restarted GMRES
// (Saddle.cu, Solvers.cu, Wrappers.cuh of the reference).
//
// Unknown x = [F^ff (6N) | S^ff (5N) | U - U_inf (6N)];
//   A x = [ M^ff x[0:11N] + (x[11N:17N]; 0) ;  x[0:6N] - R_FU x[11N:17N] ].
// Preconditioner (Saddle.cu:171-264) with M ~ I and G ~ (R_FU^pruned + relaxer D)^-1:
//   y = G (b[0:6N] - b[11N:17N]);  x = [ b[0:6N] - y ; b[6N:11N] ; y ].
// GMRES(m) is right-preconditioned, so the Givens residual is the true residual
// ||b - A x||; Arnoldi coefficients, Givens rotations and the least-squares
// solve are FP64; basis vectors are FP32.  Orthogonalisation is classical
// Gram-Schmidt with one re-orthogonalisation pass, delayed by one iteration
// so that both passes share their reads of the basis.  Everything stays on
// the device; the host polls a converged flag every few iterations.
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_solver.h"
#include "fsd_profile.h"

namespace fsd {

int saddle_multiply(fsd_handle* h, const float4* pos, const float* x, float* b, bool rebin) {
    const int N = h->p.N;
    int st = mobility_apply(h, pos, x, b, 3, x, rebin);
    if (st != FSD_OK) return st;
    lub_rfu(h, pos, x + 11 * N, b + 11 * N, x);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

__global__ void k_pc_pre(const float* __restrict__ b, float* __restrict__ t, int N) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 6 * N) t[k] = b[k] - b[11 * N + k];
}

__global__ void k_pc_post(const float* __restrict__ b, const float* __restrict__ y, float* __restrict__ x, int N) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 6 * N) {
        const float yk = y[k];
        x[k] = b[k] - yk;
        x[11 * N + k] = yk;
    } else if (k < 11 * N) {
        x[k] = b[k];
    }
}

int precond_apply(fsd_handle* h, const float* b, float* x) {
    const int N = h->p.N;
    ProfRegion pr(h, R_PRECOND_APPLY);
    if (h->p.precond == FSD_PRECOND_ICHOL) return precond_apply_ichol(h, b, x);
    if (h->p.precond == FSD_PRECOND_LEARNED) return precond_apply_learned(h, b, x);
    float* t = h->w.pc_t;
    float* y = h->w.pc_y;
    count_launch();
    k_pc_pre<<<(6 * N + 255) / 256, 256, 0, h->stream>>>(b, t, N);
    int st = precond_G(h, t, y);
    if (st != FSD_OK) return st;
    count_launch();
    k_pc_post<<<(11 * N + 255) / 256, 256, 0, h->stream>>>(b, y, x, N);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// ------------------------------------------------------------- BLAS pieces
constexpr int kRedBlocks = 296;  // two per SM
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum_d(double v, double* sh) {
    v = group_sum_d<32>(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        s = group_sum_d<32>(s);
    }
    __syncthreads();
    return s;
}

// part[i * nblocks + block] = sum over this block's slice of V_i . w, i < nv.
__global__ void __launch_bounds__(kRedThreads) k_multidot(const float* __restrict__ V, size_t ld, int nv,
                                                          const float* __restrict__ w, size_t n, double* part,
                                                          const int* done) {
    if (done && *done) return;
    __shared__ double sh[32];
    const size_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const size_t b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
    for (int i = 0; i < nv; ++i) {
        const float* vi = V + (size_t)i * ld;
        double s = 0.0;
        for (size_t k = b0 + threadIdx.x; k < b1; k += blockDim.x) s += (double)vi[k] * (double)w[k];
        s = block_sum_d(s, sh);
        if (threadIdx.x == 0) part[(size_t)i * gridDim.x + blockIdx.x] = s;
    }
}

// Same partial dots for the Gram-Schmidt passes, where nv is large: the
// block's slice of w is staged in shared memory once and each warp takes
// whole vectors, so no block-wide reduction is needed per vector.  Slices are
// `chunk` long (the launch's dynamic shared memory is chunk floats).
__global__ void __launch_bounds__(kRedThreads) k_multidot_ws(const float* __restrict__ V, size_t ld, int nv,
                                                             const float* __restrict__ w, size_t n, size_t chunk,
                                                             double* part, const int* done) {
    if (done && *done) return;
    extern __shared__ float ws[];
    const size_t b0 = (size_t)blockIdx.x * chunk;
    const size_t len = b0 < n ? min(chunk, n - b0) : 0;
    for (size_t k = threadIdx.x; k < len; k += blockDim.x) ws[k] = w[b0 + k];
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x >> 5; i < nv; i += nw) {
        const float* vi = V + (size_t)i * ld + b0;
        double s = 0.0;
        size_t k = lane;
        for (; k + 96 < len; k += 128) {
            const float a0 = vi[k], a1 = vi[k + 32], a2 = vi[k + 64], a3 = vi[k + 96];
            s += (double)a0 * ws[k] + (double)a1 * ws[k + 32] + (double)a2 * ws[k + 64] + (double)a3 * ws[k + 96];
        }
        for (; k < len; k += 32) s += (double)vi[k] * ws[k];
        s = group_sum_d<32>(s);
        if (lane == 0) part[(size_t)i * gridDim.x + blockIdx.x] = s;
    }
}

// out[i] (+)= sum_b part[i * nb + b], one warp per i.
__global__ void k_finish_dots(const double* part, int nb, int nv, double* out, bool accumulate, const int* done) {
    if (done && *done) return;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= nv) return;
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += part[(size_t)i * nb + b];
    s = group_sum_d<32>(s);
    if (lane == 0) out[i] = accumulate ? out[i] + s : s;
}

// w -= sum_i c[i] V_i.
__global__ void k_multiaxpy(const float* __restrict__ V, size_t ld, int nv, const double* __restrict__ c, float* w,
                            size_t n, const int* done) {
    if (done && *done) return;
    __shared__ float cs[kMaxRestart + 1];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) cs[i] = (float)c[i];
    __syncthreads();
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float acc = w[k];
        for (int i = 0; i < nv; ++i) acc -= cs[i] * V[(size_t)i * ld + k];
        w[k] = acc;
    }
}

// y = sum_i c[i] V_i.
__global__ void k_combine(const float* __restrict__ V, size_t ld, int nv, const double* __restrict__ c,
                          float* __restrict__ y, size_t n) {
    __shared__ float cs[kMaxRestart + 1];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) cs[i] = (float)c[i];
    __syncthreads();
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (int i = 0; i < nv; ++i) acc += cs[i] * V[(size_t)i * ld + k];
        y[k] = acc;
    }
}

__global__ void k_scale_copy(const float* __restrict__ src, float* __restrict__ dst, size_t n, const double* norm,
                             const int* done) {
    if (done && *done) return;
    const double nv = *norm;
    const float s = nv > 0.0 ? (float)(1.0 / sqrt(nv)) : 0.0f;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = src[k] * s;
}

__global__ void k_residual(const float* __restrict__ b, const float* __restrict__ Ax, float* __restrict__ r, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        r[k] = b[k] - Ax[k];
}

__global__ void k_axpy(float* __restrict__ x, const float* __restrict__ u, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        x[k] += u[k];
}

__global__ void k_add_dots(double* a, const double* b, int n, const int* done) {
    if (done && *done) return;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] += b[i];
}

// --------------------------------------------------------- Arnoldi control
// State (FP64) for one restart cycle.
constexpr int kConfirmPasses = 3;  // true-residual confirmations per solve

struct GmresState {
    double H[kMaxRestart + 1][kMaxRestart];  // column-major by iteration: H[row][col]
    double cs[kMaxRestart], sn[kMaxRestart];
    double g[kMaxRestart + 1];
    double y[kMaxRestart];
    double bnorm2;     // ||b||^2
    double beta2;      // ||r0||^2 at cycle start
    double resid;      // current relative residual estimate
    double tol;
    int j;             // completed iterations this cycle
    int total;         // total iterations
    int done;          // converged or broke down this cycle
    int breakdown;
    // Delayed re-orthogonalisation: the last column waits for the next
    // iteration's correction (pending = 1), and Tc[c][i] expresses the
    // vector that was preconditioned at iteration c in the final basis:
    // v~_c = sum_{i<=c} Tc[c][i] V_i.
    int pending;
    int nu_breakdown;
    double rscale;  // r_{j-1} was stored divided by rscale (= nu of iteration j-1)
    double Tc[kMaxRestart][kMaxRestart];
};

// Start of a cycle: r0 norm is in dots[0].
__global__ void k_cycle_start(GmresState* s, const double* dots, double tol, int first) {
    const double beta2 = dots[0];
    if (first) {
        s->total = 0;
        s->bnorm2 = dots[1];
    }
    s->tol = tol;
    s->beta2 = beta2;
    s->j = 0;
    s->breakdown = 0;
    s->pending = 0;
    s->nu_breakdown = 0;
    for (int i = 0; i <= kMaxRestart; ++i) s->g[i] = 0.0;
    s->g[0] = sqrt(beta2);
    const double bn = s->bnorm2 > 0.0 ? sqrt(s->bnorm2) : 1.0;
    s->resid = sqrt(beta2) / bn;
    s->done = (s->resid <= tol || beta2 == 0.0 || !(beta2 == beta2)) ? 1 : 0;
}

// After orthogonalising column j: h[0..j] in hcol, ||w||^2 in hcol[j+1].
__global__ void k_arnoldi_update(GmresState* s, const double* hcol, int m) {
    if (s->done) return;
    const int j = s->j;
    for (int i = 0; i <= j; ++i) s->H[i][j] = hcol[i];
    const double hn2 = hcol[j + 1];
    double hj1 = sqrt(hn2 > 0.0 ? hn2 : 0.0);
    s->H[j + 1][j] = hj1;
    for (int i = 0; i < j; ++i) {
        const double a = s->H[i][j], b = s->H[i + 1][j];
        s->H[i][j] = s->cs[i] * a + s->sn[i] * b;
        s->H[i + 1][j] = -s->sn[i] * a + s->cs[i] * b;
    }
    const double a = s->H[j][j], b = s->H[j + 1][j];
    const double r = hypot(a, b);
    const double c = r > 0.0 ? a / r : 1.0, sv = r > 0.0 ? b / r : 0.0;
    s->cs[j] = c;
    s->sn[j] = sv;
    s->H[j][j] = r;
    s->H[j + 1][j] = 0.0;
    s->g[j + 1] = -sv * s->g[j];
    s->g[j] = c * s->g[j];
    s->j = j + 1;
    s->total += 1;
    const double bn = s->bnorm2 > 0.0 ? sqrt(s->bnorm2) : 1.0;
    s->resid = fabs(s->g[j + 1]) / bn;
    if (!(hj1 > 1e-300) || !(s->resid == s->resid)) s->breakdown = (hj1 > 1e-300) ? 2 : 1;
    if (s->resid <= s->tol || s->j >= m || s->breakdown) s->done = 1;
}

// Least-squares solve H y = g (upper triangular, size j).  With apply_t the
// coefficients are mapped from the preconditioned vectors to the final basis:
// sum_c y_c v~_c = sum_i (T y)_i V_i.
__global__ void k_lsq(GmresState* s, int apply_t) {
    const int j = s->j;
    for (int i = j - 1; i >= 0; --i) {
        double v = s->g[i];
        for (int k = i + 1; k < j; ++k) v -= s->H[i][k] * s->y[k];
        s->y[i] = (s->H[i][i] != 0.0) ? v / s->H[i][i] : 0.0;
    }
    if (!apply_t) return;
    for (int i = 0; i < j; ++i) {
        double v = 0.0;
        for (int c = i; c < j; ++c) v += s->Tc[c][i] * s->y[c];
        s->y[i] = v;  // y[c] for c > i is still unmapped; y[i] is not read again
    }
}

struct GmresHost {
    int j, total, done, breakdown;
    double resid;
};

__global__ void k_export(const GmresState* s, GmresHost* o) {
    o->j = s->j;
    o->total = s->total;
    o->done = s->done;
    o->breakdown = s->breakdown;
    o->resid = s->resid;
}

// ------------------------------------------- delayed re-orthogonalisation
// Gram-Schmidt with delayed re-orthogonalisation (DCGS2: Bielich, Langou,
// Thomas, Swirydowicz, Yamazaki, Boman, Parallel Computing 2022).  Iteration
// j preconditions and multiplies the once-orthogonalised, unnormalised vector
// v~_j left in slot j by iteration j-1.  One pass reads V_0..V_j against v~_j
// and w = A M^-1 v~_j (a_i = V_i.v~_j, b_i = V_i.w, alpha = |v~_j|^2,
// beta = v~_j.w); a second pass writes the re-orthogonalised
// V_j = (v~_j - sum a_i V_i) / nu with nu^2 = alpha - sum a_i^2, and the next
// vector r_j = w - sum b_i V_i - h V_j, h = (beta - sum a_i b_i) / nu.  So the
// basis is read twice per iteration instead of four times.  r_j is stored
// divided by nu (v~_{j+1} = r_j / nu), so that the lagged vectors keep unit
// scale instead of compounding the subdiagonal entries (which underflows
// fp32 within a few dozen iterations).  Column j-1 of H is completed by
// nu_{j-1} times the a_i and nu of iteration j; column j is committed at
// once, with |r_j| below it, when its tentative residual meets the tolerance
// or the cycle is full.

// part[(2i) nb + b] = V_i . V_j and part[(2i+1) nb + b] = V_i . w over block
// b's slice, i <= j; both slices of V_j and w are staged in shared memory.
// Slices are `chunk` long, a multiple of 4, and the basis vectors start on
// 16-byte boundaries, so the basis is read as float4.
__global__ void __launch_bounds__(kRedThreads) k_dots_pair(const float* __restrict__ V, size_t ld, int j,
                                                           const float* __restrict__ w, size_t n, size_t chunk,
                                                           double* part, const int* done) {
    if (*done) return;
    extern __shared__ float4 sm4[];
    float4* sv = sm4;
    float4* sw = sm4 + chunk / 4;
    const size_t b0 = (size_t)blockIdx.x * chunk;
    const size_t len = b0 < n ? min(chunk, n - b0) : 0;
    const size_t len4 = len / 4;
    const float* vj = V + (size_t)j * ld + b0;
    for (size_t k = threadIdx.x; k < len4; k += blockDim.x) {
        sv[k] = reinterpret_cast<const float4*>(vj)[k];
        sw[k] = make_float4(w[b0 + 4 * k], w[b0 + 4 * k + 1], w[b0 + 4 * k + 2], w[b0 + 4 * k + 3]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x >> 5; i <= j; i += nw) {
        const float4* vi = reinterpret_cast<const float4*>(V + (size_t)i * ld + b0);
        double s1 = 0.0, s2 = 0.0;
        size_t k = lane;
        for (; k + 32 < len4; k += 64) {
            const float4 a = vi[k], c = vi[k + 32];
            const float4 p = sv[k], q = sw[k], p2 = sv[k + 32], q2 = sw[k + 32];
            s1 += (double)a.x * p.x + (double)a.y * p.y + (double)a.z * p.z + (double)a.w * p.w +
                  (double)c.x * p2.x + (double)c.y * p2.y + (double)c.z * p2.z + (double)c.w * p2.w;
            s2 += (double)a.x * q.x + (double)a.y * q.y + (double)a.z * q.z + (double)a.w * q.w +
                  (double)c.x * q2.x + (double)c.y * q2.y + (double)c.z * q2.z + (double)c.w * q2.w;
        }
        for (; k < len4; k += 32) {
            const float4 a = vi[k], p = sv[k], q = sw[k];
            s1 += (double)a.x * p.x + (double)a.y * p.y + (double)a.z * p.z + (double)a.w * p.w;
            s2 += (double)a.x * q.x + (double)a.y * q.y + (double)a.z * q.z + (double)a.w * q.w;
        }
        // the ragged end of the last slice
        const float* vs = V + (size_t)i * ld + b0;
        for (size_t t = 4 * len4 + lane; t < len; t += 32) {
            s1 += (double)vs[t] * vj[t];
            s2 += (double)vs[t] * w[b0 + t];
        }
        s1 = group_sum_d<32>(s1);
        s2 = group_sum_d<32>(s2);
        if (lane == 0) {
            part[(size_t)(2 * i) * gridDim.x + blockIdx.x] = s1;
            part[(size_t)(2 * i + 1) * gridDim.x + blockIdx.x] = s2;
        }
    }
}

// Givens rotations 0..c-1 applied to column col (rows 0..c, in shared
// memory) with hsub below it, then a new rotation for (c, c+1), stored in
// cs/sn[c]; g (rows c, c+1) and the residual are updated in the state.
__device__ void givens_column(double* col, int c, double hsub, double* cs, double* sn, GmresState* s) {
    col[c + 1] = hsub;
    for (int i = 0; i < c; ++i) {
        const double a = col[i], b = col[i + 1];
        col[i] = cs[i] * a + sn[i] * b;
        col[i + 1] = -sn[i] * a + cs[i] * b;
    }
    const double a = col[c], b = col[c + 1];
    const double r = hypot(a, b);
    const double cc = r > 0.0 ? a / r : 1.0, sv = r > 0.0 ? b / r : 0.0;
    cs[c] = cc;
    sn[c] = sv;
    col[c] = r;
    col[c + 1] = 0.0;
    const double gc = s->g[c];
    s->g[c + 1] = -sv * gc;
    s->g[c] = cc * gc;
    const double bn = s->bnorm2 > 0.0 ? sqrt(s->bnorm2) : 1.0;
    s->resid = fabs(s->g[c + 1]) / bn;
}

// Residual after raw column col (rows 0..c) with hsub below it, no changes.
__device__ double tentative_resid(const double* col, int c, double hsub, const double* cs, const double* sn,
                                  const GmresState* s) {
    double a = col[0];
    for (int i = 0; i < c; ++i) a = -sn[i] * a + cs[i] * col[i + 1];
    const double r = hypot(a, hsub);
    const double sv = r > 0.0 ? hsub / r : 0.0;
    const double bn = s->bnorm2 > 0.0 ? sqrt(s->bnorm2) : 1.0;
    return fabs(sv * s->g[c]) / bn;
}

// Second pass of iteration j (dots = the 2(j+1) finished sums of the first):
// V_j re-orthogonalised in place, r_j / nu written to slot j+1, its squared
// norm reduced by the last block, which then completes column j-1 and
// commits column j or leaves it pending.  Every block computes the same
// coefficients.  Only the last block touches the state after every block has
// read `done`; its serial work runs on shared-memory copies.
__global__ void __launch_bounds__(kRedThreads, 2) k_dcgs_update(float* V, size_t ld, int j, const float* __restrict__ w,
                                                             size_t n, const double* __restrict__ dots,
                                                             GmresState* s, int m, double* part, unsigned* ticket) {
    if (s->done) return;
    __shared__ float ca[kMaxRestart + 1], cc[kMaxRestart + 1];
    __shared__ double sh[2][32];
    __shared__ double s_nu, s_h;
    double a2 = 0.0, ab = 0.0;
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
        const double a = dots[2 * i], b = dots[2 * i + 1];
        a2 += a * a;
        ab += a * b;
    }
    a2 = group_sum_d<32>(a2);
    ab = group_sum_d<32>(ab);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = a2;
        sh[1][wid] = ab;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double A2 = 0.0, AB = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            A2 += sh[0][q];
            AB += sh[1][q];
        }
        const double nu2 = dots[2 * j] - A2;
        const double nu = nu2 > 0.0 ? sqrt(nu2) : 0.0;
        s_nu = nu;
        s_h = nu > 0.0 ? (dots[2 * j + 1] - AB) / nu : 0.0;
    }
    __syncthreads();
    const double nu = s_nu, hj = s_h;
    const double hn = nu > 0.0 ? hj / nu : 0.0;
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
        const double a = dots[2 * i], b = dots[2 * i + 1];
        ca[i] = (float)a;
        cc[i] = (float)(b - hn * a);
    }
    __syncthreads();
    const float fv = nu > 0.0 ? (float)(1.0 / nu) : 0.f;
    const float fh = (float)hn;
    float4* vj = reinterpret_cast<float4*>(V + (size_t)j * ld);
    float4* vn = reinterpret_cast<float4*>(V + (size_t)(j + 1) * ld);
    const float4* w4 = reinterpret_cast<const float4*>(w);
    const bool w_aligned = (reinterpret_cast<uintptr_t>(w) & 15) == 0;
    const size_t n4 = (n + 3) / 4;  // the basis stride is padded to 32 floats; w is read element-wise at its end
    double sig = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n4; k += (size_t)gridDim.x * blockDim.x) {
        const float4 vt = vj[k];
        float4 aw;
        if (w_aligned && 4 * k + 3 < n) {
            aw = w4[k];
        } else {
            aw.x = 4 * k < n ? w[4 * k] : 0.f;
            aw.y = 4 * k + 1 < n ? w[4 * k + 1] : 0.f;
            aw.z = 4 * k + 2 < n ? w[4 * k + 2] : 0.f;
            aw.w = 4 * k + 3 < n ? w[4 * k + 3] : 0.f;
        }
        float4 av = vt;
        for (int i = 0; i < j; ++i) {
            const float4 vi = reinterpret_cast<const float4*>(V + (size_t)i * ld)[k];
            const float a = ca[i], c = cc[i];
            av.x = fmaf(-a, vi.x, av.x);
            av.y = fmaf(-a, vi.y, av.y);
            av.z = fmaf(-a, vi.z, av.z);
            av.w = fmaf(-a, vi.w, av.w);
            aw.x = fmaf(-c, vi.x, aw.x);
            aw.y = fmaf(-c, vi.y, aw.y);
            aw.z = fmaf(-c, vi.z, aw.z);
            aw.w = fmaf(-c, vi.w, aw.w);
        }
        float4 r;
        r.x = fmaf(-fh, vt.x, aw.x) * fv;
        r.y = fmaf(-fh, vt.y, aw.y) * fv;
        r.z = fmaf(-fh, vt.z, aw.z) * fv;
        r.w = fmaf(-fh, vt.w, aw.w) * fv;
        float4 v = make_float4(av.x * fv, av.y * fv, av.z * fv, av.w * fv);
        if (4 * k + 3 >= n) {  // padding past 17N stays zero (it was never written before)
            if (4 * k + 1 >= n) r.y = v.y = 0.f;
            if (4 * k + 2 >= n) r.z = v.z = 0.f;
            r.w = v.w = 0.f;
        }
        vj[k] = v;
        vn[k] = r;
        sig += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z + (double)r.w * r.w;
    }
    block_partial(sig, part);
    if (!last_block(ticket)) return;
    __shared__ double cprev[kMaxRestart + 2], ccur[kMaxRestart + 2], scs[kMaxRestart + 1], ssn[kMaxRestart + 1];
    __shared__ int commit, drop_j, pend_s;
    const bool pend = j > 0 && s->pending;
    const double rs = s->rscale;
    for (int i = threadIdx.x; i <= j; i += blockDim.x) {
        if (i < j) {
            scs[i] = s->cs[i];
            ssn[i] = s->sn[i];
            if (pend) cprev[i] = s->H[i][j - 1] + rs * dots[2 * i];
            s->Tc[j][i] = dots[2 * i];
        } else {
            s->Tc[j][j] = nu;
        }
        ccur[i] = i < j ? dots[2 * i + 1] : hj;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const double sum = warp_sum_parts(part, gridDim.x);
        if (threadIdx.x == 0) {
            s->total += 1;
            if (pend) givens_column(cprev, j - 1, rs * nu, scs, ssn, s);
            pend_s = pend;
            commit = 0;
            drop_j = 0;
            const double hsub = nu * sqrt(sum);
            s->rscale = nu;
            s->pending = 0;
            if (!(nu > 1e-300)) {  // v~_j lay in the span of V_0..V_j-1
                s->breakdown = 1;
                s->j = j;
                s->done = 1;
                drop_j = 1;
            } else {
                s->j = j + 1;
                const double rt = tentative_resid(ccur, j, hsub, scs, ssn, s);
                const bool bad = !(hsub > 1e-300) || !(rt == rt);
                if (rt <= s->tol || j + 1 >= m || bad) {
                    givens_column(ccur, j, hsub, scs, ssn, s);
                    if (bad) s->breakdown = (hsub > 1e-300) ? 2 : 1;
                    s->done = 1;
                    commit = 1;
                } else {
                    s->pending = 1;
                }
            }
            *ticket = 0;
        }
    }
    __syncthreads();
    // Write back: column j-1 rotated, column j rotated (committed) or raw (pending).
    for (int i = threadIdx.x; i <= j + 1; i += blockDim.x) {
        if (pend_s && i <= j) s->H[i][j - 1] = cprev[i];
        if (!drop_j && (i <= j || commit)) s->H[i][j] = ccur[i];
        if (pend_s && i == j - 1) {
            s->cs[i] = scs[i];
            s->sn[i] = ssn[i];
        }
        if (commit && i == j) {
            s->cs[i] = scs[i];
            s->sn[i] = ssn[i];
        }
    }
}

static const double* gs_y(const GmresState* s) {
    return reinterpret_cast<const double*>(reinterpret_cast<const char*>(s) + offsetof(GmresState, y));
}

int gmres_alloc(fsd_handle* h) {
    FSD_CHECK_CUDA(cudaMalloc(&h->w.gmres_state, sizeof(GmresState)));
    FSD_CHECK_CUDA(cudaMallocHost(&h->w.gmres_host, sizeof(GmresHost)));
    return FSD_OK;
}

// Solve A x = b; x holds the initial guess.  Returns FSD_OK or
// FSD_ERR_GMRES_MAXIT / FSD_ERR_BREAKDOWN; iterations and the final true
// relative residual in *iters / *resid.
int saddle_solve(fsd_handle* h, const float4* pos, const float* b, float* x, float tol, int* iters, float* resid) {
    Workspace& w = h->w;
    const int N = h->p.N;
    const size_t n = (size_t)17 * N;
    const int m = std::min(h->p.gmres_restart, kMaxRestart);
    const int maxit = h->p.gmres_max_iter;
    cudaStream_t st = h->stream;
    GmresState* gs = (GmresState*)w.gmres_state;
    GmresHost* gh = (GmresHost*)w.gmres_host;
    const size_t ld = krylov_ld(N);
    float* V = w.V;
    float* r = w.sx;   // residual / work
    float* Ax = w.sy;  // operator output
    float* z = w.sz;   // preconditioned vector
    double* part = w.dred;
    double* dots = w.hcol;  // [0..m+1]
    const int nbl = kRedBlocks;
    const int vthreads = 256, vblocks = 4 * 148;
    // Flexible GMRES (Saad 1993) when the preconditioner varies between
    // applications: the preconditioned basis Z is kept and x += Z y.
    const bool flexible = precond_is_flexible(h);
    if (flexible && !w.Z) return FSD_ERR_BAD_PARAMS;
    const size_t chunk = (n + nbl - 1) / nbl;
    const bool staged = chunk * sizeof(float) <= 48 * 1024;
    // Delayed re-orthogonalisation stages two slices per block, each a
    // multiple of 4 floats long.
    const size_t chunk4 = (chunk + 3) & ~(size_t)3;
    const size_t pair_smem = 2 * chunk4 * sizeof(float);
    const bool delayed = pair_smem <= 200 * 1024;
    if (delayed && pair_smem > 48 * 1024)
        FSD_CHECK_CUDA(ensure_smem_limit((const void*)k_dots_pair, pair_smem));
    auto multidot = [&](const float* Vb, size_t ldv, int nv, const float* wv, size_t nn, double* pt, const int* dn) {
        if (staged)
            k_multidot_ws<<<nbl, kRedThreads, chunk * sizeof(float), st>>>(Vb, ldv, nv, wv, nn, chunk, pt, dn);
        else
            k_multidot<<<nbl, kRedThreads, 0, st>>>(Vb, ldv, nv, wv, nn, pt, dn);
    };
    int total = 0;
    bool first = true;
    int status = FSD_OK;
    double rel = 0.0;
    // The Arnoldi residual estimate drifts from the true residual once the
    // FP32 basis loses orthogonality; a solve whose true residual is still
    // above tol restarts from it (at most kConfirmPasses times).
    for (int pass = 0; pass < kConfirmPasses; ++pass) {
        status = FSD_OK;
        // ||b||^2 into dots[1] (first cycle only).
        for (;;) {
            // r = b - A x
            int e = saddle_multiply(h, pos, x, Ax, first);
            if (e != FSD_OK) return e;
            count_launch();
            k_residual<<<vblocks, vthreads, 0, st>>>(b, Ax, r, n);
            count_launch();
            k_multidot<<<nbl, kRedThreads, 0, st>>>(r, n, 1, r, n, part, nullptr);
            count_launch();
            k_finish_dots<<<1, 32, 0, st>>>(part, nbl, 1, dots, false, nullptr);
            if (first) {
                count_launch();
                k_multidot<<<nbl, kRedThreads, 0, st>>>(b, n, 1, b, n, part, nullptr);
                count_launch();
                k_finish_dots<<<1, 32, 0, st>>>(part, nbl, 1, dots + 1, false, nullptr);
            }
            count_launch();
            k_cycle_start<<<1, 1, 0, st>>>(gs, dots, (double)tol, first ? 1 : 0);
            count_launch();
            k_scale_copy<<<vblocks, vthreads, 0, st>>>(r, V, n, dots, &gs->done);
            first = false;
            count_launch();
            k_export<<<1, 1, 0, st>>>(gs, gh);
            FSD_CHECK_CUDA(cudaStreamSynchronize(st));
            const bool converged_at_start = gh->done != 0;
            for (int j = 0; j < m && !converged_at_start; ++j) {
                // w = A M^-1 V_j
                float* zj = flexible ? w.Z + (size_t)j * ld : z;
                e = precond_apply(h, V + (size_t)j * ld, zj);
                if (e != FSD_OK) return e;
                e = saddle_multiply(h, pos, zj, Ax, false);
                if (e != FSD_OK) return e;
                ProfRegion pk(h, R_KRYLOV);
                if (delayed) {
                    count_launch();
                    k_dots_pair<<<nbl, kRedThreads, pair_smem, st>>>(V, ld, j, Ax, n, chunk4, part, &gs->done);
                    count_launch();
                    k_finish_dots<<<(2 * (j + 1) + 7) / 8, 256, 0, st>>>(part, nbl, 2 * (j + 1), dots, false,
                                                                         &gs->done);
                    count_launch();
                    k_dcgs_update<<<2 * 148, kRedThreads, 0, st>>>(V, ld, j, Ax, n, dots, gs, m, part, w.ticket);
                    if ((j % 4) == 3 || j == m - 1) {
                        count_launch();
                        k_export<<<1, 1, 0, st>>>(gs, gh);
                        FSD_CHECK_CUDA(cudaStreamSynchronize(st));
                        if (gh->done) break;
                    }
                    continue;
                }
                // CGS2 against V_0..V_j.
                count_launch();
                multidot(V, ld, j + 1, Ax, n, part, &gs->done);
                count_launch();
                k_finish_dots<<<(j + 1 + 7) / 8, 256, 0, st>>>(part, nbl, j + 1, dots, false, &gs->done);
                count_launch();
                k_multiaxpy<<<vblocks, vthreads, 0, st>>>(V, ld, j + 1, dots, Ax, n, &gs->done);
                count_launch();
                multidot(V, ld, j + 1, Ax, n, part, &gs->done);
                count_launch();
                k_finish_dots<<<(j + 1 + 7) / 8, 256, 0, st>>>(part, nbl, j + 1, w.hcol2, false, &gs->done);
                count_launch();
                k_multiaxpy<<<vblocks, vthreads, 0, st>>>(V, ld, j + 1, w.hcol2, Ax, n, &gs->done);
                count_launch();
                k_add_dots<<<1, 128, 0, st>>>(dots, w.hcol2, j + 1, &gs->done);
                count_launch();
                k_multidot<<<nbl, kRedThreads, 0, st>>>(Ax, n, 1, Ax, n, part, &gs->done);
                count_launch();
                k_finish_dots<<<1, 32, 0, st>>>(part, nbl, 1, dots + j + 1, false, &gs->done);
                count_launch();
                k_arnoldi_update<<<1, 1, 0, st>>>(gs, dots, m);
                count_launch();
                k_scale_copy<<<vblocks, vthreads, 0, st>>>(Ax, V + (size_t)(j + 1) * ld, n, dots + j + 1, &gs->done);
                if ((j % 4) == 3 || j == m - 1) {
                    count_launch();
                    k_export<<<1, 1, 0, st>>>(gs, gh);
                    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
                    if (gh->done) break;
                }
            }
            count_launch();
            k_export<<<1, 1, 0, st>>>(gs, gh);
            FSD_CHECK_CUDA(cudaStreamSynchronize(st));
            if (getenv("FSD_DEBUG_GMRES"))
                fprintf(stderr, "gmres cycle: j=%d total=%d resid=%.3e breakdown=%d\n", gh->j, gh->total, gh->resid,
                        gh->breakdown);
            const int jc = gh->j;
            total = gh->total;
            if (jc > 0) {
                count_launch();
                k_lsq<<<1, 1, 0, st>>>(gs, delayed && !flexible ? 1 : 0);
                if (flexible) {  // x += Z y
                    count_launch();
                    k_combine<<<vblocks, vthreads, 0, st>>>(w.Z, ld, jc, gs_y(gs), z, n);
                } else {  // x += M^-1 V y
                    count_launch();
                    k_combine<<<vblocks, vthreads, 0, st>>>(V, ld, jc, gs_y(gs), Ax, n);
                    e = precond_apply(h, Ax, z);
                    if (e != FSD_OK) return e;
                }
                count_launch();
                k_axpy<<<vblocks, vthreads, 0, st>>>(x, z, n);
            }
            if (gh->breakdown == 1) {
                status = FSD_ERR_BREAKDOWN;
                break;
            }
            if (gh->resid <= tol && jc < m) break;  // converged inside the cycle; confirm below
            if (gh->resid <= tol) break;
            if (total >= maxit) {
                status = FSD_ERR_GMRES_MAXIT;
                break;
            }
        }
        // True residual of the returned solution.
        int e = saddle_multiply(h, pos, x, Ax, false);
        if (e != FSD_OK) return e;
        count_launch();
        k_residual<<<vblocks, vthreads, 0, st>>>(b, Ax, r, n);
        count_launch();
        k_multidot<<<nbl, kRedThreads, 0, st>>>(r, n, 1, r, n, part, nullptr);
        count_launch();
        k_finish_dots<<<1, 32, 0, st>>>(part, nbl, 1, dots, false, nullptr);
        double host[2];
        FSD_CHECK_CUDA(cudaMemcpyAsync(host, dots, sizeof(double), cudaMemcpyDeviceToHost, st));
        FSD_CHECK_CUDA(cudaMemcpyAsync(host + 1, &gs->bnorm2, sizeof(double), cudaMemcpyDeviceToHost, st));
        FSD_CHECK_CUDA(cudaStreamSynchronize(st));
        rel = host[1] > 0 ? sqrt(host[0] / host[1]) : sqrt(host[0]);
        if (status != FSD_OK || !(rel > tol) || total >= maxit) break;
    }
    const int ws = precond_wait_status(h);
    if (ws != FSD_OK) return ws;
    if (iters) *iters = total;
    if (resid) *resid = (float)rel;
    if (!(rel == rel)) status = FSD_ERR_BREAKDOWN;
    // Above tolerance after the restarts from the true residual (the FP32 floor
    // lies near 1e-7 relative) or at the iteration limit: not converged.
    if (status == FSD_OK && rel > tol) status = FSD_ERR_GMRES_MAXIT;
    return status;
}

}  // namespace fsd
