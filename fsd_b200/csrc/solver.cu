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
// Gram-Schmidt with one re-orthogonalisation pass.  Everything stays on the
// device; the host polls a converged flag every few iterations.
#include <cmath>
#include <cstddef>
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

// Least-squares solve H y = g (upper triangular, size j).
__global__ void k_lsq(GmresState* s) {
    const int j = s->j;
    for (int i = j - 1; i >= 0; --i) {
        double v = s->g[i];
        for (int k = i + 1; k < j; ++k) v -= s->H[i][k] * s->y[k];
        s->y[i] = (s->H[i][i] != 0.0) ? v / s->H[i][i] : 0.0;
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
    const size_t ld = n;
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
                // CGS2 against V_0..V_j.
                ProfRegion pk(h, R_KRYLOV);
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
                k_lsq<<<1, 1, 0, st>>>(gs);
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
