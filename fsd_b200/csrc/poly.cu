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

// Block-CSR copy of A and the row tiles of G and A for the streamed
// products (bsr_tma.cu), once per build.
int poly_prepare_products(fsd_handle* h) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    std::vector<unsigned> pn(N);
    std::vector<int> grow(N + 1), arow(N + 1);
    FSD_CHECK_CUDA(cudaMemcpyAsync(pn.data(), s->a_pn, sizeof(unsigned) * N, cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(grow.data(), s->g_rowptr, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    arow[0] = 0;
    for (int i = 0; i < N; ++i) arow[i + 1] = arow[i] + (int)pn[i];
    const size_t nnz = (size_t)arow[N];
    if (!s->a_rowptr) FSD_CHECK_CUDA(cudaMalloc(&s->a_rowptr, sizeof(int) * (N + 1)));
    if (nnz + 8 > s->a_cap) {  // headroom: the column copy reads up to three past the end
        if (s->a_col) cudaFree(s->a_col);
        if (s->a_val) cudaFree(s->a_val);
        s->a_col = nullptr;
        s->a_val = nullptr;
        const size_t cap = nnz + nnz / 8 + 1024;
        FSD_CHECK_CUDA(cudaMalloc(&s->a_col, sizeof(int) * cap));
        FSD_CHECK_CUDA(cudaMalloc(&s->a_val, sizeof(float) * 36 * cap));
        s->a_cap = cap;
    }
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->a_rowptr, arow.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));
    count_launch();
    k_compact_pruned<<<(N + 7) / 8, 256, 0, st>>>(s->a_pn, s->a_plist, s->a_blocks, s->a_rowptr, N, s->a_col,
                                                  s->a_val);
    std::vector<int> gt, at;
    int e = bsr_make_tiles(grow, N, gt);
    if (e != FSD_OK) return e;
    e = bsr_make_tiles(arow, N, at);
    if (e != FSD_OK) return e;
    if (!s->g_tiles) {
        s->tile_cap = N / 3 + 2;  // a full tile holds >= 3 rows (> 72 of at most 104 blocks, rows <= 32)
        FSD_CHECK_CUDA(cudaMalloc(&s->g_tiles, sizeof(int) * (s->tile_cap + 2)));
        FSD_CHECK_CUDA(cudaMalloc(&s->a_tiles, sizeof(int) * (s->tile_cap + 2)));
        e = bsr_tma_prepare();
        if (e != FSD_OK) return e;
    }
    const int ng = (int)gt.size() - 1, na = (int)at.size() - 1;
    if (ng > s->tile_cap || na > s->tile_cap) return FSD_ERR_BAD_PARAMS;
    gt.resize(s->tile_cap + 1, N);
    at.resize(s->tile_cap + 1, N);
    gt.push_back(ng);
    at.push_back(na);
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->g_tiles, gt.data(), sizeof(int) * (s->tile_cap + 2), cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->a_tiles, at.data(), sizeof(int) * (s->tile_cap + 2), cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));  // the host tile vectors go out of scope
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Clenshaw slots: b_{k-1} in slot 0; each b_m goes to the slot that holds
// neither b_{m+1} nor b_{m+2}.
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

static BsrTmaArgs g_args(const LearnedState* s, int N) {
    BsrTmaArgs a{};
    a.rowptr = s->g_rowptr;
    a.col = s->g_col;
    a.val = s->g_val;
    a.tile_row = s->g_tiles;
    a.ntiles = s->g_tiles + s->tile_cap + 1;
    a.N = N;
    a.pc = s->pc;
    return a;
}

static BsrTmaArgs a_args(const LearnedState* s, int N) {
    BsrTmaArgs a{};
    a.rowptr = s->a_rowptr;
    a.col = s->a_col;
    a.val = s->a_val;
    a.tile_row = s->a_tiles;
    a.ntiles = s->a_tiles + s->tile_cap + 1;
    a.N = N;
    a.pc = s->pc;
    return a;
}

// Arguments of the first (mode 0) and last (mode 2) products for b and x.
static BsrTmaArgs first_args(const LearnedState* s, int N, int k, const float* b) {
    const size_t n6 = 6 * (size_t)N;
    BsrTmaArgs a = g_args(s, N);
    a.x = b;
    a.T = s->pbuf;
    a.out = s->pbuf + n6;
    a.B = s->pbuf + 2 * n6;
    a.k = k;
    return a;
}

static BsrTmaArgs last_args(const LearnedState* s, int N, int k, const float* b, float* x) {
    const size_t n6 = 6 * (size_t)N;
    BsrTmaArgs a = g_args(s, N);
    a.x = s->pbuf + (2 + poly_v_slot(k)) * n6;
    a.b = b;
    a.xs = x;
    return a;
}

// Kernels of one application on b into x, enqueued on st (for capture):
// k products with G and k - 1 with A.
static int poly_enqueue(fsd_handle* h, const float* b, float* x, cudaStream_t st) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    const int k = h->p.learned_poly;
    const size_t n6 = 6 * (size_t)N;
    const int grid = s->tile_cap;
    float* T = s->pbuf;
    float* U = s->pbuf + n6;
    float* Bs[3] = {s->pbuf + 2 * n6, s->pbuf + 3 * n6, s->pbuf + 4 * n6};
    bsr_tma_launch(0, first_args(s, N, k, b), grid, st);  // U = c_{k-1} G t, b_{k-1} -> slot 0
    int cur = 0, prev = -1;
    for (int m = k - 2; m >= 0; --m) {
        if (m < k - 2) {
            BsrTmaArgs ga = g_args(s, N);
            ga.x = Bs[cur];
            ga.out = U;
            bsr_tma_launch(1, ga, grid, st);
        }
        const int nxt = poly_next_slot(cur, prev);
        BsrTmaArgs aa = a_args(s, N);
        aa.x = U;
        aa.T = T;
        aa.B1 = Bs[cur];
        aa.B2 = prev >= 0 ? Bs[prev] : nullptr;
        aa.m = m;
        aa.out = Bs[nxt];
        bsr_tma_launch(3, aa, grid, st);
        prev = cur;
        cur = nxt;
    }
    bsr_tma_launch(2, last_args(s, N, k, b, x), grid, st);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

static int poly_kernels(int k) { return 2 * k - 1; }

static int poly_graph(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    const void* key[12] = {s->g_rowptr, s->g_col, s->g_val, s->a_rowptr, s->a_col,  s->a_val,
                           s->g_tiles,  s->a_tiles, s->pbuf, s->pc,       nullptr,   nullptr};
    bool same = s->pexec && s->pkey_k == h->p.learned_poly;
    for (int i = 0; i < 10 && same; ++i) same = key[i] == s->pkey[i];
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
        if (kp.func == bsr_tma_kernel(0)) s->pnode_first = nd;
        if (kp.func == bsr_tma_kernel(2)) s->pnode_last = nd;
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
    for (int i = 0; i < 10; ++i) s->pkey[i] = key[i];
    s->pkey_k = h->p.learned_poly;
    return FSD_OK;
}

// Point the first node at b and the last at (b, x).
static int poly_bind(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    const int N = h->p.N, k = h->p.learned_poly;
    BsrTmaArgs fa = first_args(s, N, k, b), la = last_args(s, N, k, b, x);
    void* fargs[] = {&fa};
    void* largs[] = {&la};
    cudaKernelNodeParams kp = {};
    kp.gridDim = dim3(s->tile_cap);
    kp.blockDim = dim3(kBsrThreads);
    kp.sharedMemBytes = (unsigned)bsr_tma_smem();
    kp.func = (void*)bsr_tma_kernel(0);
    kp.kernelParams = fargs;
    FSD_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(s->pexec, s->pnode_first, &kp));
    kp.func = (void*)bsr_tma_kernel(2);
    kp.kernelParams = largs;
    FSD_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(s->pexec, s->pnode_last, &kp));
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

// Coefficients of q for the Chebyshev interval [rho lambda, lambda]: the
// residual polynomial 1 - x q(x) = T_k((1 + rho - 2u)/(1 - rho)) /
// T_k((1 + rho)/(1 - rho)), u = x / lambda, is the classical Chebyshev
// acceleration on that interval (bounded by one on all of [0, lambda], so no
// eigenvalue of AG is amplified, and smallest on [rho lambda, lambda]).  q has
// degree k - 1 and is expanded exactly in T_m(2u - 1), m < k, by Chebyshev
// interpolation at k nodes (FP64).
static double cheb_T(int n, double z) {
    if (std::fabs(z) <= 1.0) return std::cos(n * std::acos(z));
    const double v = std::cosh(n * std::acosh(std::fabs(z)));
    return (z < 0 && (n & 1)) ? -v : v;
}

void poly_interval_coefficients(double rho, double lambda, int k, float* c) {
    const double zs = (1.0 + rho) / (1.0 - rho);
    const double Tz = cheb_T(k, zs);
    std::vector<double> gu(k), uu(k);
    for (int j = 0; j < k; ++j) {
        const double th = M_PI * (j + 0.5) / k;
        const double u = 0.5 * (std::cos(th) + 1.0);
        const double r = cheb_T(k, (1.0 + rho - 2.0 * u) / (1.0 - rho)) / Tz;
        uu[j] = u;
        gu[j] = (1.0 - r) / (lambda * u);
    }
    for (int m = 0; m < k; ++m) {
        double acc = 0.0;
        for (int j = 0; j < k; ++j) acc += gu[j] * std::cos(m * M_PI * (j + 0.5) / k);
        c[m] = (float)((m == 0 ? 1.0 : 2.0) * acc / k);
    }
}

// Coefficients for the interval ratio rho (in (0, 1)) with the spectral
// bound of the last power iteration; caller's stream, synchronised.
int poly_set_interval(fsd_handle* h, double rho) {
    LearnedState* s = learned(h);
    const int k = h->p.learned_poly;
    float pc[kMaxPoly + 1];
    FSD_CHECK_CUDA(cudaMemcpyAsync(pc, s->pc, sizeof(float) * (kMaxPoly + 1), cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    const double lambda = pc[kMaxPoly];
    if (!(lambda > 0.0) || !(rho > 0.0 && rho < 1.0)) return FSD_ERR_BREAKDOWN;
    float c[kMaxPoly] = {};
    poly_interval_coefficients(rho, lambda, k, c);
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->pc, c, sizeof(float) * kMaxPoly, cudaMemcpyHostToDevice, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    s->poly_ratio = (float)rho;
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
    s->user_ratio = -1.f;
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
    void* ptrs[] = {s->pc, s->pbuf, s->ppart, s->pnrm, s->pticket, s->a_rowptr, s->a_col, s->a_val, s->g_tiles,
                    s->a_tiles};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->pexec) cudaGraphExecDestroy(s->pexec);
    if (s->pgraph) cudaGraphDestroy(s->pgraph);
}

}  // namespace fsd
