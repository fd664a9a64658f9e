// Block-sparse preconditioner slot G for FSD_PRECOND_LEARNED.
//
// G ~ (R_FU^pruned + relaxer D)^-1 is an explicit block-sparse matrix
// (6x6 fp32 blocks in block-CSR over particles, original particle order), so
// one application is a single parallel SpMV instead of the two sequential
// triangular solves of the IC(0) factor.  The blocks are produced by the
// message-passing network at each preconditioner build, or set directly through
// fsd_precond_set_blocks.  The saddle pre/post steps (Saddle.cu:171-264) are
// fused into the SpMV kernel, exactly as in the IC(0) solve kernels.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_profile.h"
#include "fsd_solver.h"

namespace fsd {

LearnedState* learned(fsd_handle* h) {
    if (!h->learned) h->learned = new LearnedState();
    return (LearnedState*)h->learned;
}

void learned_free(fsd_handle* h) {
    LearnedState* s = (LearnedState*)h->learned;
    if (!s) return;
    mpnn_free(h);
    void* ptrs[] = {s->g_rowptr, s->g_col, s->g_val, s->t, s->w, s->y, s->Vi, s->Zi, s->part, s->H,
                    s->sp_sets, s->sp_size, s->sp_rowptr, s->sp_scan, s->sp_bucket, s->sp_cnt};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->sp_host) cudaFreeHost(s->sp_host);
    if (s->tb) cudaFree(s->tb);
    if (s->tx) cudaFree(s->tx);
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
    delete s;
    h->learned = nullptr;
}

// Grow the block-CSR storage of G to hold nnzb blocks.
int learned_reserve(fsd_handle* h, int nnzb) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    if (!s->g_rowptr) FSD_CHECK_CUDA(cudaMalloc(&s->g_rowptr, sizeof(int) * (N + 1)));
    if (nnzb > s->g_cap) {
        if (s->g_col) cudaFree(s->g_col);
        if (s->g_val) cudaFree(s->g_val);
        s->g_col = nullptr;
        s->g_val = nullptr;
        s->g_cap = 0;
        // headroom, so that pattern growth from step to step rarely reallocates
        const int cap = nnzb + nnzb / 8 + 1024;
        FSD_CHECK_CUDA(cudaMalloc(&s->g_col, sizeof(int) * (size_t)cap));
        FSD_CHECK_CUDA(cudaMalloc(&s->g_val, sizeof(float) * 36 * (size_t)cap));
        s->g_cap = cap;
    }
    return FSD_OK;
}

// Copy a caller's block-CSR G after checking its structure on the host, so
// that no kernel ever indexes outside the vectors it reads.
int learned_set_blocks(fsd_handle* h, int nnzb, const int* d_rowptr, const int* d_col, const float* d_val) {
    const int N = h->p.N;
    if (nnzb < 0) return FSD_ERR_BAD_PARAMS;
    std::vector<int> rp(N + 1), cl((size_t)nnzb);
    FSD_CHECK_CUDA(cudaMemcpyAsync(rp.data(), d_rowptr, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost, h->stream));
    if (nnzb)
        FSD_CHECK_CUDA(
            cudaMemcpyAsync(cl.data(), d_col, sizeof(int) * (size_t)nnzb, cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (rp[0] != 0 || rp[N] != nnzb) return FSD_ERR_BAD_PARAMS;
    for (int i = 0; i < N; ++i)
        if (rp[i + 1] < rp[i]) return FSD_ERR_BAD_PARAMS;
    for (int c : cl)
        if (c < 0 || c >= N) return FSD_ERR_BAD_PARAMS;
    const int e = learned_reserve(h, nnzb);
    if (e != FSD_OK) return e;
    LearnedState* s = learned(h);
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->g_rowptr, d_rowptr, sizeof(int) * (N + 1), cudaMemcpyDeviceToDevice, h->stream));
    if (nnzb) {
        FSD_CHECK_CUDA(cudaMemcpyAsync(s->g_col, d_col, sizeof(int) * (size_t)nnzb, cudaMemcpyDeviceToDevice,
                                       h->stream));
        FSD_CHECK_CUDA(cudaMemcpyAsync(s->g_val, d_val, sizeof(float) * 36 * (size_t)nnzb, cudaMemcpyDeviceToDevice,
                                       h->stream));
    }
    s->g_nnzb = nnzb;
    s->g_user = true;
    return FSD_OK;
}

// x = P^-1 b with y = G t, t_i = b[6i:6i+6] - b[11N+6i:11N+6i+6]:
// x[6i:6i+6] = b[6i:6i+6] - y_i, x[6N:11N] = b[6N:11N], x[11N+6i:...] = y_i.
// Eight lanes per particle row; lane r < 6 owns output component r.
__global__ void __launch_bounds__(256) k_pc_bsr(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                const float* __restrict__ G, const float* __restrict__ b,
                                                float* __restrict__ x, int N) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;  // whole groups of eight leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const float* bU = b + 11 * (size_t)N;
    float acc = 0.f;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
        const int j = col[e];
        const float tj = (r < 6) ? b[6 * j + r] - bU[6 * j + r] : 0.f;
        const float* Ge = G + (size_t)e * 36 + (r < 6 ? r : 0) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float tc = __shfl_sync(gmask, tj, c, 8);
            if (r < 6) acc += Ge[c] * tc;
        }
    }
    if (r < 6) {
        x[6 * i + r] = b[6 * i + r] - acc;
        x[11 * (size_t)N + 6 * i + r] = acc;
    }
    if (r < 5) x[6 * (size_t)N + 5 * i + r] = b[6 * (size_t)N + 5 * i + r];
}

// ----------------------------------------------------------- inner solve
// y = sum_s A_is x_s over the pruned list (self included), 8 lanes per row.
__global__ void __launch_bounds__(256) k_pruned_spmv(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                                                     const float* __restrict__ A, const float* __restrict__ x,
                                                     float* __restrict__ y, int N) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    float acc = 0.f;
    const unsigned n = pn[i];
    for (unsigned s = 0; s < n; ++s) {
        const size_t e = (size_t)i * kPrunedCap + s;
        const unsigned j = plist[e];
        const float xj = (r < 6) ? x[6 * j + r] : 0.f;
        const float* Ae = A + e * 36 + (r < 6 ? r : 0) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float xc = __shfl_sync(gmask, xj, c, 8);
            if (r < 6) acc += Ae[c] * xc;
        }
    }
    if (r < 6) y[6 * i + r] = acc;
}

// y = G x in block CSR.
__global__ void __launch_bounds__(256) k_bsr_spmv(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const float* __restrict__ G, const float* __restrict__ x,
                                                  float* __restrict__ y, int N) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    float acc = 0.f;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
        const int j = col[e];
        const float xj = (r < 6) ? x[6 * j + r] : 0.f;
        const float* Ge = G + (size_t)e * 36 + (r < 6 ? r : 0) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float xc = __shfl_sync(gmask, xj, c, 8);
            if (r < 6) acc += Ge[c] * xc;
        }
    }
    if (r < 6) y[6 * i + r] = acc;
}

constexpr int kInnerBlocks = 296;
constexpr int kInnerThreads = 256;

// t = b[0:6N] - b[11N:17N]; part[b] = partial ||t||^2.
__global__ void __launch_bounds__(kInnerThreads) k_inner_rhs(const float* __restrict__ b, float* __restrict__ t,
                                                             int N, double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 6 * N; k += gridDim.x * blockDim.x) {
        const float v = b[k] - b[11 * (size_t)N + k];
        t[k] = v;
        s += (double)v * v;
    }
    s = group_sum_d<32>(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        v = group_sum_d<32>(v);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

// part[i * nb + block] = V_i . w over the block's grid-stride share, i < nv.
__global__ void __launch_bounds__(kInnerThreads) k_inner_dots(const float* __restrict__ V, size_t ld, int nv,
                                                              const float* __restrict__ w, size_t n, double* part) {
    __shared__ double sh[kMaxInner + 1][kInnerThreads / 32];
    double acc[kMaxInner + 1];
#pragma unroll
    for (int i = 0; i <= kMaxInner; ++i) acc[i] = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const double wk = w[k];
#pragma unroll
        for (int i = 0; i <= kMaxInner; ++i)
            if (i < nv) acc[i] += (double)V[(size_t)i * ld + k] * wk;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i <= kMaxInner; ++i) {
        if (i >= nv) break;
        const double v = group_sum_d<32>(acc[i]);
        if (lane == 0) sh[i][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double v = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += sh[threadIdx.x][q];
        part[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
}

// H[col j][i] = sum_b part[i * nb + b] for i < nv (one warp per i).  With
// j < 0 the single sum is the squared norm of the right-hand side, kept in
// H's beta slot.
__global__ void k_inner_finish(const double* part, int nb, int nv, double* H, int j) {
    const int i = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (i >= nv) return;
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += part[(size_t)i * nb + b];
    s = group_sum_d<32>(s);
    if (lane == 0) {
        if (j < 0) H[(kMaxInner + 1) * kMaxInner] = s;
        else H[(size_t)j * (kMaxInner + 1) + i] = s;
    }
}

// w -= sum_{i<nv} H[j][i] V_i, and part[b] = partial ||w||^2.
__global__ void __launch_bounds__(kInnerThreads) k_inner_orth(const float* __restrict__ V, size_t ld, int nv,
                                                              const double* __restrict__ H, int j, float* w, size_t n,
                                                              double* part) {
    __shared__ float hc[kMaxInner + 1];
    __shared__ double sh[32];
    if (threadIdx.x < nv) hc[threadIdx.x] = (float)H[(size_t)j * (kMaxInner + 1) + threadIdx.x];
    __syncthreads();
    double s = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float acc = w[k];
        for (int i = 0; i < nv; ++i) acc -= hc[i] * V[(size_t)i * ld + k];
        w[k] = acc;
        s += (double)acc * acc;
    }
    s = group_sum_d<32>(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        v = group_sum_d<32>(v);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

// dst = src / sqrt(nrm2) with nrm2 = sum of part (every block re-reduces the
// few partials, so no extra launch is needed); the norm is written to
// H[j][j+1] (j >= 0) or to the beta slot (j < 0).  A zero norm gives zero.
__global__ void __launch_bounds__(kInnerThreads) k_inner_scale(const float* __restrict__ src, float* __restrict__ dst,
                                                               size_t n, const double* __restrict__ part, int nb,
                                                               double* H, int j) {
    __shared__ double sh[32];
    __shared__ double nrm;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
    s = group_sum_d<32>(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += sh[q];
        nrm = sqrt(v);
        if (blockIdx.x == 0) {
            if (j < 0) H[(kMaxInner + 1) * kMaxInner] = nrm;
            else H[(size_t)j * (kMaxInner + 1) + j + 1] = nrm;
        }
    }
    __syncthreads();
    const float f = nrm > 0.0 ? (float)(1.0 / nrm) : 0.0f;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = f * src[k];
}

// Least squares min || beta e1 - H y || by Givens rotations in FP64 (one
// thread; k <= kMaxInner).  Columns after a breakdown (zero subdiagonal or
// zero pivot) are dropped.  y is written to H's last column block.
__global__ void k_inner_lsq(double* H, int k) {
    if (threadIdx.x != 0) return;
    double R[kMaxInner + 1][kMaxInner];
    double g[kMaxInner + 1];
    const double beta = H[(kMaxInner + 1) * kMaxInner];
    for (int c = 0; c < k; ++c)
        for (int r = 0; r <= k; ++r) R[r][c] = H[(size_t)c * (kMaxInner + 1) + r];
    for (int r = 0; r <= k; ++r) g[r] = 0.0;
    g[0] = beta;
    int used = k;
    for (int c = 0; c < k; ++c) {
        const double a = R[c][c], bb = R[c + 1][c];
        const double rr = sqrt(a * a + bb * bb);
        if (!(rr > 1e-300 * (beta > 0 ? beta : 1.0))) {
            used = c;
            break;
        }
        const double cs = a / rr, sn = bb / rr;
        for (int q = c; q < k; ++q) {
            const double x0 = R[c][q], x1 = R[c + 1][q];
            R[c][q] = cs * x0 + sn * x1;
            R[c + 1][q] = -sn * x0 + cs * x1;
        }
        const double g0 = g[c], g1 = g[c + 1];
        g[c] = cs * g0 + sn * g1;
        g[c + 1] = -sn * g0 + cs * g1;
        if (!(R[c + 1][c] == R[c + 1][c])) {
            used = c;
            break;
        }
    }
    double y[kMaxInner];
    for (int c = used - 1; c >= 0; --c) {
        double v = g[c];
        for (int q = c + 1; q < used; ++q) v -= R[c][q] * y[q];
        y[c] = v / R[c][c];
    }
    double* out = H + (size_t)(kMaxInner + 1) * kMaxInner + 1;
    for (int c = 0; c < kMaxInner; ++c) out[c] = (c < used) ? y[c] : 0.0;
}

// x = post(b, sum_j c_j Z_j): x[0:6N] = b - y, x[6N:11N] = b, x[11N:] = y.
__global__ void k_inner_post(const float* __restrict__ Z, size_t ld, int k, const double* __restrict__ c,
                             const float* __restrict__ b, float* __restrict__ x, int N) {
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    if (kk < 6 * N) {
        float acc = 0.f;
        for (int i = 0; i < k; ++i) acc += (float)c[i] * Z[(size_t)i * ld + kk];
        x[kk] = b[kk] - acc;
        x[11 * (size_t)N + kk] = acc;
    } else if (kk < 11 * N) {
        x[kk] = b[kk];
    }
}

static int inner_alloc(fsd_handle* h) {
    LearnedState* s = learned(h);
    if (s->inner_cap >= 0) return FSD_OK;
    const size_t n6 = 6 * (size_t)h->p.N;
    FSD_CHECK_CUDA(cudaMalloc(&s->t, sizeof(float) * n6));
    FSD_CHECK_CUDA(cudaMalloc(&s->w, sizeof(float) * n6));
    FSD_CHECK_CUDA(cudaMalloc(&s->y, sizeof(float) * n6));
    FSD_CHECK_CUDA(cudaMalloc(&s->Vi, sizeof(float) * n6 * (kMaxInner + 1)));
    FSD_CHECK_CUDA(cudaMalloc(&s->Zi, sizeof(float) * n6 * kMaxInner));
    FSD_CHECK_CUDA(cudaMalloc(&s->part, sizeof(double) * (kMaxInner + 2) * kInnerBlocks));
    FSD_CHECK_CUDA(cudaMalloc(&s->H, sizeof(double) * ((kMaxInner + 1) * kMaxInner + 1 + kMaxInner)));
    FSD_CHECK_CUDA(cudaMalloc(&s->tb, sizeof(float) * 17 * (size_t)h->p.N));
    FSD_CHECK_CUDA(cudaMalloc(&s->tx, sizeof(float) * 17 * (size_t)h->p.N));
    s->inner_cap = kMaxInner;
    return FSD_OK;
}

bool precond_is_flexible(const fsd_handle* h) {
    return h->p.precond == FSD_PRECOND_LEARNED && h->p.learned_inner > 0;
}

// Kernels of one inner solve, enqueued on st (also used for graph capture).
static int inner_enqueue(fsd_handle* h, const float* b, float* x, cudaStream_t st) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    const int k = h->p.learned_inner;
    const size_t n6 = 6 * (size_t)N;
    const int rows = (8 * N + 255) / 256;
    const int nb = kInnerBlocks;
    k_inner_rhs<<<nb, kInnerThreads, 0, st>>>(b, s->t, N, s->part);
    k_inner_scale<<<nb, kInnerThreads, 0, st>>>(s->t, s->Vi, n6, s->part, nb, s->H, -1);
    for (int j = 0; j < k; ++j) {
        float* vj = s->Vi + (size_t)j * n6;
        float* zj = s->Zi + (size_t)j * n6;
        k_bsr_spmv<<<rows, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, vj, zj, N);
        k_pruned_spmv<<<rows, 256, 0, st>>>(s->a_pn, s->a_plist, s->a_blocks, zj, s->w, N);
        k_inner_dots<<<nb, kInnerThreads, 0, st>>>(s->Vi, n6, j + 1, s->w, n6, s->part);
        k_inner_finish<<<1, 32 * (j + 1), 0, st>>>(s->part, nb, j + 1, s->H, j);
        k_inner_orth<<<nb, kInnerThreads, 0, st>>>(s->Vi, n6, j + 1, s->H, j, s->w, n6, s->part);
        k_inner_scale<<<nb, kInnerThreads, 0, st>>>(s->w, s->Vi + (size_t)(j + 1) * n6, n6, s->part, nb, s->H, j);
    }
    k_inner_lsq<<<1, 32, 0, st>>>(s->H, k);
    k_inner_post<<<(11 * N + 255) / 256, 256, 0, st>>>(s->Zi, n6, k, s->H + (size_t)(kMaxInner + 1) * kMaxInner + 1,
                                                       b, x, N);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

static int inner_kernels(int k) { return 4 + 6 * k; }

// (Re)capture the inner solve when the arrays it reads were reallocated or k changed.
static int inner_graph(fsd_handle* h) {
    LearnedState* s = learned(h);
    const void* key[8] = {s->g_rowptr, s->g_col, s->g_val, s->a_pn, s->a_plist, s->a_blocks, s->Vi, s->Zi};
    bool same = s->gexec && s->gkey_k == h->p.learned_inner;
    for (int i = 0; i < 8 && same; ++i) same = key[i] == s->gkey[i];
    if (same) return FSD_OK;
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    s->gexec = nullptr;
    if (!s->cap_stream) FSD_CHECK_CUDA(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    FSD_CHECK_CUDA(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int e = inner_enqueue(h, s->tb, s->tx, s->cap_stream);
    const cudaError_t ce = cudaStreamEndCapture(s->cap_stream, &g);
    if (e != FSD_OK) {
        if (g) cudaGraphDestroy(g);
        return e;
    }
    FSD_CHECK_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&s->gexec, g, 0);
    cudaGraphDestroy(g);
    FSD_CHECK_CUDA(ie);
    for (int i = 0; i < 8; ++i) s->gkey[i] = key[i];
    s->gkey_k = h->p.learned_inner;
    s->captures += 1;
    if (getenv("FSD_DEBUG_GRAPH")) fprintf(stderr, "inner graph captured (%d)\n", s->captures);
    return FSD_OK;
}

// x = P^-1 b.  Without inner steps G is applied once (fused with the saddle
// pre/post steps).  With k inner steps, y ~ (R_FU^pruned + D)^-1 t comes from
// k steps of GMRES on that matrix from a zero guess, right-preconditioned by
// G; the map b -> x then depends on b nonlinearly, which the flexible outer
// GMRES allows.  The inner solve is one CUDA graph launch between a copy of b
// in and a copy of x out; no host synchronisation.
int precond_apply_learned(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    const int k = h->p.learned_inner;
    if (k == 0) {
        count_launch();
        k_pc_bsr<<<(8 * N + 255) / 256, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, b, x, N);
        FSD_CHECK_CUDA(cudaGetLastError());
        return FSD_OK;
    }
    const int e = inner_graph(h);
    if (e != FSD_OK) return e;
    const size_t n17 = 17 * (size_t)N;
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->tb, b, sizeof(float) * n17, cudaMemcpyDeviceToDevice, st));
    FSD_CHECK_CUDA(cudaGraphLaunch(s->gexec, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(x, s->tx, sizeof(float) * n17, cudaMemcpyDeviceToDevice, st));
    for (int i = 0; i < inner_kernels(k); ++i) count_launch();
    return FSD_OK;
}

// Blocks set through fsd_precond_set_blocks are used as given.  Otherwise G
// is the two-hop sparse approximate inverse of the pruned matrix, plus the
// loaded network's correction on the same pattern.
int precond_build_learned(fsd_handle* h, const float4* pos) {
    LearnedState* s = learned(h);
    ProfRegion pr(h, R_PRECOND_BUILD);
    int e = FSD_OK;
    if (h->p.learned_inner > 0) e = inner_alloc(h);
    if (e != FSD_OK) return e;
    e = precond_assemble_pruned(h, pos, 1.0f, &s->a_pn, &s->a_plist, &s->a_blocks);
    if (e != FSD_OK) return e;
    if (!s->g_user) {
        e = spai_build(h);
        if (e != FSD_OK) return e;
        if (mpnn_loaded(h)) {
            e = mpnn_infer(h, pos, s->a_pn, s->a_plist, s->a_blocks);
            if (e != FSD_OK) return e;
        }
    }
    h->pc_valid = true;
    return FSD_OK;
}

int learned_set_weights(fsd_handle* h, const float* host_w, int n) {
    const int e = mpnn_set_weights(h, host_w, n);
    if (e == FSD_OK) learned(h)->g_user = false;
    return e;
}

}  // namespace fsd
