// Learned Chebyshev polynomial inner solve of FSD_PRECOND_LEARNED.
//
// The saddle preconditioner (Saddle.cu:171-264) needs y ~ A^-1 t for the
// lubrication block A = R_FU^pruned + D.  Here
//   y = G q(AG) t,   q(x) = sum_{m<k} c_m T_m(2x/lambda - 1),
// with G the two-hop sparse approximate inverse of A (spai.cu), T_m the
// Chebyshev polynomials, lambda an upper bound of the spectrum of AG (power
// iteration when the preconditioner is built, times 1.1), and coefficients c
// that the message-passing network predicts for each configuration (mpnn.cu,
// the mean over particles of its node head) or that the caller sets.
// q(AG) t is evaluated by Clenshaw's recurrence with S = (2/lambda) AG - I:
//   b_{k-1} = c_{k-1} t,
//   b_m = c_m t + 2 S b_{m+1} - b_{m+2}        m = k-2 .. 1,
//   v = c_0 t + S b_1 - b_2,
// so one application costs k products with G, k-1 with A and no reductions.
// The map t -> y is linear and fixed within a solve, so the outer GMRES keeps
// no flexible basis.  The 2k-1 kernels are replayed from a CUDA graph whose
// first and last nodes (the only ones that touch b and x) are re-pointed at
// each application's vectors.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fsd_brownian.h"
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_profile.h"
#include "fsd_solver.h"

namespace fsd {

namespace {

constexpr int kPowerIters = 12;      // power iterations for the spectral bound
constexpr float kLambdaMargin = 1.1f;
constexpr int kRedBlocksP = 296;

// Row r of a 6x6 block times the 6-vector held by lanes 0..5 of the group.
__device__ __forceinline__ float blk_row(const float* blk, int rr, float xj, unsigned gmask) {
    const float2* g = reinterpret_cast<const float2*>(blk + rr * 6);
    const float2 g01 = g[0], g23 = g[1], g45 = g[2];
    float s = g01.x * __shfl_sync(gmask, xj, 0, 8);
    s = fmaf(g01.y, __shfl_sync(gmask, xj, 1, 8), s);
    s = fmaf(g23.x, __shfl_sync(gmask, xj, 2, 8), s);
    s = fmaf(g23.y, __shfl_sync(gmask, xj, 3, 8), s);
    s = fmaf(g45.x, __shfl_sync(gmask, xj, 4, 8), s);
    s = fmaf(g45.y, __shfl_sync(gmask, xj, 5, 8), s);
    return s;
}

// (G x)_i row component r; with FROM_B the operand is x_j = b[6j+r] - b[11N+6j+r].
template <bool FROM_B>
__device__ __forceinline__ float g_row(const int* __restrict__ rowptr, const int* __restrict__ col,
                                       const float* __restrict__ G, const float* __restrict__ x, size_t offU, int i,
                                       int r, unsigned gmask) {
    const int rr = r < 6 ? r : 0;
    auto ld = [&](int j) -> float {
        if (r >= 6) return 0.f;
        if (FROM_B) return x[6 * j + r] - x[offU + 6 * j + r];
        return x[6 * j + r];
    };
    float acc = 0.f;
    const int e1 = rowptr[i + 1];
    int e = rowptr[i];
    for (; e + 3 < e1; e += 4) {  // four blocks in flight per lane
        const int j0 = col[e], j1 = col[e + 1], j2 = col[e + 2], j3 = col[e + 3];
        const float x0 = ld(j0), x1 = ld(j1), x2 = ld(j2), x3 = ld(j3);
        const float* Ge = G + (size_t)e * 36;
        acc += blk_row(Ge, rr, x0, gmask);
        acc += blk_row(Ge + 36, rr, x1, gmask);
        acc += blk_row(Ge + 72, rr, x2, gmask);
        acc += blk_row(Ge + 108, rr, x3, gmask);
    }
    for (; e < e1; ++e) acc += blk_row(G + (size_t)e * 36, rr, ld(col[e]), gmask);
    return acc;
}

// (A x)_i row component r over the pruned list (self included).
__device__ __forceinline__ float a_row(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                                       const float* __restrict__ A, const float* __restrict__ x, int i, int r,
                                       unsigned gmask) {
    const int rr = r < 6 ? r : 0;
    const unsigned n = pn[i];
    const size_t e0 = (size_t)i * kPrunedCap;
    float acc = 0.f;
    unsigned q = 0;
    for (; q + 3 < n; q += 4) {
        const unsigned j0 = plist[e0 + q], j1 = plist[e0 + q + 1], j2 = plist[e0 + q + 2], j3 = plist[e0 + q + 3];
        const float x0 = r < 6 ? x[6 * j0 + r] : 0.f, x1 = r < 6 ? x[6 * j1 + r] : 0.f;
        const float x2 = r < 6 ? x[6 * j2 + r] : 0.f, x3 = r < 6 ? x[6 * j3 + r] : 0.f;
        const float* Ae = A + (e0 + q) * 36;
        acc += blk_row(Ae, rr, x0, gmask);
        acc += blk_row(Ae + 36, rr, x1, gmask);
        acc += blk_row(Ae + 72, rr, x2, gmask);
        acc += blk_row(Ae + 108, rr, x3, gmask);
    }
    for (; q < n; ++q) {
        const unsigned j = plist[e0 + q];
        acc += blk_row(A + (e0 + q) * 36, rr, r < 6 ? x[6 * j + r] : 0.f, gmask);
    }
    return acc;
}

// u = c_{k-1} G t with t = b[0:6N] - b[11N:17N]; T = t and B = c_{k-1} t (own row).
__global__ void __launch_bounds__(256) k_poly_first(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                    const float* __restrict__ G, const float* __restrict__ b,
                                                    const float* __restrict__ pc, int k, int N, float* __restrict__ T,
                                                    float* __restrict__ B, float* __restrict__ U) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;  // whole groups of eight leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const size_t offU = 11 * (size_t)N;
    const float c = pc[k - 1];
    const float acc = g_row<true>(rowptr, col, G, b, offU, i, r, gmask);
    if (r < 6) {
        const float t = b[6 * i + r] - b[offU + 6 * i + r];
        T[6 * i + r] = t;
        B[6 * i + r] = c * t;
        U[6 * i + r] = c * acc;
    }
}

// U = G X.
__global__ void __launch_bounds__(256) k_poly_g(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                const float* __restrict__ G, const float* __restrict__ X, int N,
                                                float* __restrict__ U) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const float acc = g_row<false>(rowptr, col, G, X, 0, i, r, gmask);
    if (r < 6) U[6 * i + r] = acc;
}

// out = c_m T + f ((2/lambda) A U - B1) - B2 (B2 may be null), f = 2 for m >= 1
// and 1 for m = 0 (Clenshaw's last step).
__global__ void __launch_bounds__(256) k_poly_a(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                                                const float* __restrict__ A, const float* __restrict__ U,
                                                const float* __restrict__ T, const float* __restrict__ B1,
                                                const float* __restrict__ B2, const float* __restrict__ pc, int m,
                                                int N, float* __restrict__ out) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const float acc = a_row(pn, plist, A, U, i, r, gmask);
    if (r < 6) {
        const size_t q = 6 * (size_t)i + r;
        const float s2 = 2.0f / pc[kMaxPoly];
        const float f = m >= 1 ? 2.0f : 1.0f;
        float v = fmaf(pc[m], T[q], f * fmaf(s2, acc, -B1[q]));
        if (B2) v -= B2[q];
        out[q] = v;
    }
}

// y = G V; x = [b[0:6N] - y ; b[6N:11N] ; y].
__global__ void __launch_bounds__(256) k_poly_last(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                   const float* __restrict__ G, const float* __restrict__ V,
                                                   const float* b, float* x, int N) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const float y = g_row<false>(rowptr, col, G, V, 0, i, r, gmask);
    if (r < 6) {
        const size_t q = 6 * (size_t)i + r;
        const float bq = b[q];
        x[q] = bq - y;
        x[11 * (size_t)N + q] = y;
    }
    if (r < 5) {
        const size_t q = 6 * (size_t)N + 5 * (size_t)i + r;
        x[q] = b[q];
    }
}

// ---------------------------------------------------------- spectral bound
__global__ void k_set_double(double* p, double v) { *p = v; }

// W = A U, |W| into nrm[0] and kLambdaMargin |W| into pc[kMaxPoly] by the last block.
__global__ void __launch_bounds__(256) k_power_a(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                                                 const float* __restrict__ A, const float* __restrict__ U, int N,
                                                 float* __restrict__ W, double* part, unsigned* ticket, double* nrm,
                                                 float* pc) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int r = threadIdx.x & 7;
    double s = 0.0;
    if (i < N) {  // whole groups of eight; every thread reaches the reduction
        const unsigned gmask = 0xffu << (threadIdx.x & 24);
        const float acc = a_row(pn, plist, A, U, i, r, gmask);
        if (r < 6) {
            W[6 * i + r] = acc;
            s = (double)acc * acc;
        }
    }
    block_partial(s, part);
    if (!last_block(ticket)) return;
    if (threadIdx.x < 32) {
        const double t = sqrt(warp_sum_parts(part, gridDim.x));
        if (threadIdx.x == 0) {
            nrm[0] = t;
            pc[kMaxPoly] = (float)(kLambdaMargin * t);
            *ticket = 0;
        }
    }
}

// U = G (W / nrm[0]).
__global__ void __launch_bounds__(256) k_power_g(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                 const float* __restrict__ G, const float* __restrict__ W,
                                                 const double* __restrict__ nrm, int N, float* __restrict__ U) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const float acc = g_row<false>(rowptr, col, G, W, 0, i, r, gmask);
    const double nv = *nrm;
    const float f = nv > 0.0 ? (float)(1.0 / nv) : 0.f;
    if (r < 6) U[6 * i + r] = f * acc;
}

}  // namespace

int poly_alloc(fsd_handle* h) {
    LearnedState* s = learned(h);
    if (s->pc) return FSD_OK;
    const size_t n6 = 6 * (size_t)h->p.N;
    FSD_CHECK_CUDA(cudaMalloc(&s->pc, sizeof(float) * (kMaxPoly + 1)));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->pc, 0, sizeof(float) * (kMaxPoly + 1), h->stream));
    FSD_CHECK_CUDA(cudaMalloc(&s->pbuf, sizeof(float) * n6 * 5));
    FSD_CHECK_CUDA(cudaMalloc(&s->ppart, sizeof(double) * std::max<size_t>(kRedBlocksP, (8 * n6 / 6 + 255) / 256)));
    FSD_CHECK_CUDA(cudaMalloc(&s->pnrm, sizeof(double) * 2));
    FSD_CHECK_CUDA(cudaMalloc(&s->pticket, sizeof(unsigned)));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->pticket, 0, sizeof(unsigned), h->stream));
    return FSD_OK;
}

bool poly_active(const fsd_handle* h) {
    return h->p.precond == FSD_PRECOND_LEARNED && h->p.learned_poly >= 2;
}

// Upper bound of the spectrum of AG into pc[kMaxPoly]: kPowerIters power
// iterations from a fixed counter-based start vector, times 1.1.
int poly_lambda(fsd_handle* h) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    const size_t n6 = 6 * (size_t)N;
    cudaStream_t st = h->stream;
    float* W = s->pbuf;
    float* U = s->pbuf + n6;
    const int rows = (8 * N + 255) / 256;
    gaussian(h, W, n6, 1, kStreamGain, 1.0f);
    count_launch();
    k_set_double<<<1, 1, 0, st>>>(s->pnrm, std::sqrt((double)n6));
    for (int it = 0; it < kPowerIters; ++it) {
        count_launch();
        k_power_g<<<rows, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, W, s->pnrm, N, U);
        count_launch();
        k_power_a<<<rows, 256, 0, st>>>(s->a_pn, s->a_plist, s->a_blocks, U, N, W, s->ppart, s->pticket, s->pnrm,
                                        s->pc);
    }
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Clenshaw slots: b_{k-1} in slot 0; each b_m goes to the slot that holds
// neither b_{m+1} nor b_{m+2}.  Returns the slot of b_m and updates (cur, prev).
static int poly_next_slot(int cur, int prev) { return (cur + 1) % 3 == prev ? (cur + 2) % 3 : (cur + 1) % 3; }

// Slot that holds v = b_0 after the recurrence for k coefficients.
static int poly_v_slot(int k) {
    int cur = 0, prev = -1;
    for (int m = k - 2; m >= 0; --m) {
        const int nxt = poly_next_slot(cur, prev);
        prev = cur;
        cur = nxt;
    }
    return cur;
}

// Kernels of one application on b into x, enqueued on st (for capture).
static int poly_enqueue(fsd_handle* h, const float* b, float* x, cudaStream_t st) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    const int k = h->p.learned_poly;
    const size_t n6 = 6 * (size_t)N;
    const int rows = (8 * N + 255) / 256;
    float* T = s->pbuf;
    float* U = s->pbuf + n6;
    float* Bs[3] = {s->pbuf + 2 * n6, s->pbuf + 3 * n6, s->pbuf + 4 * n6};
    // b_{k-1} -> Bs[0]; then b_m into the slot after b_{m+1}
    k_poly_first<<<rows, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, b, s->pc, k, N, T, Bs[0], U);
    int cur = 0;           // slot of b_{m+1}
    int prev = -1;         // slot of b_{m+2} (none for m = k-2)
    for (int m = k - 2; m >= 0; --m) {
        if (m < k - 2) k_poly_g<<<rows, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, Bs[cur], N, U);
        const int nxt = poly_next_slot(cur, prev);
        k_poly_a<<<rows, 256, 0, st>>>(s->a_pn, s->a_plist, s->a_blocks, U, T, Bs[cur], prev >= 0 ? Bs[prev] : nullptr,
                                       s->pc, m, N, Bs[nxt]);
        prev = cur;
        cur = nxt;
    }
    k_poly_last<<<rows, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, Bs[cur], b, x, N);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

static int poly_kernels(int k) { return 2 * k - 1; }

static int poly_graph(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    const void* key[8] = {s->g_rowptr, s->g_col, s->g_val, s->a_pn, s->a_plist, s->a_blocks, s->pbuf, s->pc};
    bool same = s->pexec && s->pkey_k == h->p.learned_poly;
    for (int i = 0; i < 8 && same; ++i) same = key[i] == s->pkey[i];
    if (same) return FSD_OK;
    if (s->pexec) cudaGraphExecDestroy(s->pexec);
    if (s->pgraph) cudaGraphDestroy(s->pgraph);
    s->pexec = nullptr;
    s->pgraph = nullptr;
    if (!s->cap_stream) FSD_CHECK_CUDA(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    FSD_CHECK_CUDA(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int e = poly_enqueue(h, b, x, s->cap_stream);
    const cudaError_t ce = cudaStreamEndCapture(s->cap_stream, &g);
    if (e != FSD_OK) {
        if (g) cudaGraphDestroy(g);
        return e;
    }
    FSD_CHECK_CUDA(ce);
    size_t nn = 0;
    FSD_CHECK_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    FSD_CHECK_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    s->pnode_first = s->pnode_last = nullptr;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        FSD_CHECK_CUDA(cudaGraphNodeGetType(nd, &t));
        if (t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        FSD_CHECK_CUDA(cudaGraphKernelNodeGetParams(nd, &kp));
        if (kp.func == (void*)k_poly_first) s->pnode_first = nd;
        if (kp.func == (void*)k_poly_last) s->pnode_last = nd;
    }
    if (!s->pnode_first || !s->pnode_last) {
        cudaGraphDestroy(g);
        return FSD_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&s->pexec, g, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        FSD_CHECK_CUDA(ie);
    }
    s->pgraph = g;
    for (int i = 0; i < 8; ++i) s->pkey[i] = key[i];
    s->pkey_k = h->p.learned_poly;
    return FSD_OK;
}

// Point the first node at b and the last at (b, x).
static int poly_bind(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    int N = h->p.N;
    int k = h->p.learned_poly;
    const size_t n6 = 6 * (size_t)N;
    const int rows = (8 * N + 255) / 256;
    const int* rowptr = s->g_rowptr;
    const int* col = s->g_col;
    const float* G = s->g_val;
    const float* pc = s->pc;
    float* T = s->pbuf;
    float* U = s->pbuf + n6;
    float* B0 = s->pbuf + 2 * n6;
    void* first_args[] = {&rowptr, &col, &G, &b, &pc, &k, &N, &T, &B0, &U};
    cudaKernelNodeParams kf = {};
    kf.func = (void*)k_poly_first;
    kf.gridDim = dim3(rows);
    kf.blockDim = dim3(256);
    kf.kernelParams = first_args;
    FSD_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(s->pexec, s->pnode_first, &kf));
    const float* V = s->pbuf + (2 + poly_v_slot(k)) * n6;  // the Clenshaw slot that holds v
    void* last_args[] = {&rowptr, &col, &G, &V, &b, &x, &N};
    cudaKernelNodeParams kl = {};
    kl.func = (void*)k_poly_last;
    kl.gridDim = dim3(rows);
    kl.blockDim = dim3(256);
    kl.kernelParams = last_args;
    FSD_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(s->pexec, s->pnode_last, &kl));
    return FSD_OK;
}

int poly_apply(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    int e = poly_graph(h, b, x);
    if (e != FSD_OK) return e;
    e = poly_bind(h, b, x);
    if (e != FSD_OK) return e;
    FSD_CHECK_CUDA(cudaGraphLaunch(s->pexec, h->stream));
    for (int i = 0; i < poly_kernels(h->p.learned_poly); ++i) count_launch();
    return FSD_OK;
}

int poly_set_coefficients(fsd_handle* h, const float* host_c, int k) {
    if (k < 2 || k > kMaxPoly || !host_c) return FSD_ERR_BAD_PARAMS;
    const int e = poly_alloc(h);
    if (e != FSD_OK) return e;
    LearnedState* s = learned(h);
    float c[kMaxPoly] = {};
    for (int m = 0; m < k; ++m) c[m] = host_c[m];
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->pc, c, sizeof(float) * kMaxPoly, cudaMemcpyHostToDevice, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    s->poly_user = true;
    return FSD_OK;
}

int poly_get_coefficients(fsd_handle* h, float* host_c, int n) {
    LearnedState* s = learned(h);
    if (!host_c || n < kMaxPoly + 1 || !s->pc) return FSD_ERR_BAD_PARAMS;
    FSD_CHECK_CUDA(cudaMemcpyAsync(host_c, s->pc, sizeof(float) * (kMaxPoly + 1), cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return FSD_OK;
}

void poly_free(LearnedState* s) {
    void* ptrs[] = {s->pc, s->pbuf, s->ppart, s->pnrm, s->pticket};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->pexec) cudaGraphExecDestroy(s->pexec);
    if (s->pgraph) cudaGraphDestroy(s->pgraph);
}

}  // namespace fsd
