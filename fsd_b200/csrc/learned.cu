// Block-sparse preconditioner slot G for FSD_PRECOND_LEARNED.
//
// G ~ (R_FU^pruned + relaxer D)^-1 is an explicit block-sparse matrix (6x6
// fp32 blocks in block-CSR over particles, original particle order): the
// two-hop sparse approximate inverse of the pruned matrix (spai.cu), plus the
// loaded network's correction (mpnn.cu), or blocks set directly through
// fsd_precond_set_blocks.  Applied once (learned_inner = 0, fused with the
// saddle pre/post steps of Saddle.cu:171-264) or as the right preconditioner
// of a few inner GMRES steps on the pruned matrix itself, replayed from a
// CUDA graph.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
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
    void* ptrs[] = {s->g_rowptr, s->g_col,   s->g_val,     s->Vi,        s->Zi,        s->part,   s->H,
                    s->nrm,      s->ticket,  s->sp_sets,   s->sp_size,   s->sp_rowptr, s->sp_scan, s->sp_bucket,
                    s->sp_cnt};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->sp_host) cudaFreeHost(s->sp_host);
    poly_free(s);
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->graph) cudaGraphDestroy(s->graph);
    if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
    delete s;
    h->learned = nullptr;
}

// Grow the block-CSR storage of G to hold nnzb blocks.
int learned_reserve(fsd_handle* h, int nnzb) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    if (!s->g_rowptr) FSD_CHECK_CUDA(cudaMalloc(&s->g_rowptr, sizeof(int) * (N + 1)));
    if (nnzb + 8 > s->g_cap) {  // headroom: the streamed products read column indices up to three past the end
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
// The blocks stay fp32: the lubrication blocks are ill-conditioned (gaps down
// to 1e-3), and fp16 copies, even scaled per block, raised the outer
// iteration counts by a quarter.

// Row r of a 6x6 fp32 block times x, summed over a group of eight lanes
// (lane c < 6 holds x_c in xj).
__device__ __forceinline__ float block_row(const float* blk, int rr, float xj, unsigned gmask) {
    const float2* g = reinterpret_cast<const float2*>(blk + rr * 6);
    const float2 g01 = g[0], g23 = g[1], g45 = g[2];
    float sum = g01.x * __shfl_sync(gmask, xj, 0, 8);
    sum = fmaf(g01.y, __shfl_sync(gmask, xj, 1, 8), sum);
    sum = fmaf(g23.x, __shfl_sync(gmask, xj, 2, 8), sum);
    sum = fmaf(g23.y, __shfl_sync(gmask, xj, 3, 8), sum);
    sum = fmaf(g45.x, __shfl_sync(gmask, xj, 4, 8), sum);
    sum = fmaf(g45.y, __shfl_sync(gmask, xj, 5, 8), sum);
    return sum;
}

// z = G (u / |u|) in block CSR, |u| read from the device (zero gives zero).
// Eight lanes per particle row; lane r < 6 owns output component r.
__global__ void __launch_bounds__(256) k_bsr_spmv_n(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                    const float* __restrict__ G, const float* __restrict__ u,
                                                    const double* __restrict__ unrm, float* __restrict__ z, int N) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = threadIdx.x & 7;
    const int i = gid >> 3;  // rows in storage order: the kernel streams G
    if (i >= N) return;      // whole groups of eight leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const int rr = r < 6 ? r : 0;
    float acc = 0.f;
    const int e1 = rowptr[i + 1];
    int e = rowptr[i];
    for (; e + 3 < e1; e += 4) {  // four blocks in flight per lane
        const int j0 = col[e], j1 = col[e + 1], j2 = col[e + 2], j3 = col[e + 3];
        const float x0 = (r < 6) ? u[6 * j0 + r] : 0.f, x1 = (r < 6) ? u[6 * j1 + r] : 0.f;
        const float x2 = (r < 6) ? u[6 * j2 + r] : 0.f, x3 = (r < 6) ? u[6 * j3 + r] : 0.f;
        const float* Ge = G + (size_t)e * 36;
        acc += block_row(Ge, rr, x0, gmask);
        acc += block_row(Ge + 36, rr, x1, gmask);
        acc += block_row(Ge + 72, rr, x2, gmask);
        acc += block_row(Ge + 108, rr, x3, gmask);
    }
    for (; e < e1; ++e) {
        const int j = col[e];
        const float xj = (r < 6) ? u[6 * j + r] : 0.f;
        acc += block_row(G + (size_t)e * 36, rr, xj, gmask);
    }
    const double nv = *unrm;
    const float f = nv > 0.0 ? (float)(1.0 / nv) : 0.f;
    if (r < 6) z[6 * i + r] = f * acc;
}

constexpr int kInnerBlocks = 296;
constexpr int kInnerThreads = 256;

// u0 = b[0:6N] - b[11N:17N]; |u0| goes to nrm[0] and to H's beta slot.
__global__ void __launch_bounds__(kInnerThreads) k_inner_rhs(const float* __restrict__ b, float* __restrict__ u0,
                                                             int N, double* part, unsigned* ticket, double* H,
                                                             double* nrm) {
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 6 * N; k += gridDim.x * blockDim.x) {
        const float v = b[k] - b[11 * (size_t)N + k];
        u0[k] = v;
        s += (double)v * v;
    }
    block_partial(s, part);
    if (!last_block(ticket)) return;
    if (threadIdx.x < 32) {
        const double t = sqrt(warp_sum_parts(part, gridDim.x));
        if (threadIdx.x == 0) {
            nrm[0] = t;
            H[(kMaxInner + 1) * kMaxInner] = t;
            *ticket = 0;
        }
    }
}

// w = A z over the pruned list (self included), written to the basis slot
// U_nv, fused with the dots H[j][q] = (U_q . w) / |U_q| for q < nv = j + 1.
__global__ void __launch_bounds__(256) k_pruned_spmv_dots(const unsigned* __restrict__ pn,
                                                          const unsigned* __restrict__ plist,
                                                          const float* __restrict__ A,
                                                          const float* __restrict__ z, float* U, size_t ld, int nv,
                                                          const double* __restrict__ nrm, double* part,
                                                          unsigned* ticket, double* H, int j, int N) {
    __shared__ double sh[kMaxInner + 1][8];
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 3;  // rows in storage order: the kernel streams A
    const bool row_ok = i < N;
    const int r = threadIdx.x & 7;
    const bool act = row_ok && r < 6;
    float acc = 0.f;
    if (row_ok) {  // whole groups of eight; every thread reaches the reductions below
        const unsigned gmask = 0xffu << (threadIdx.x & 24);
        const int rr = r < 6 ? r : 0;
        const unsigned n = pn[i];
        const size_t e0 = (size_t)i * kPrunedCap;
        unsigned q = 0;
        for (; q + 3 < n; q += 4) {  // four blocks in flight per lane
            const unsigned j0 = plist[e0 + q], j1 = plist[e0 + q + 1], j2 = plist[e0 + q + 2], j3 = plist[e0 + q + 3];
            const float x0 = (r < 6) ? z[6 * j0 + r] : 0.f, x1 = (r < 6) ? z[6 * j1 + r] : 0.f;
            const float x2 = (r < 6) ? z[6 * j2 + r] : 0.f, x3 = (r < 6) ? z[6 * j3 + r] : 0.f;
            const float* Ae = A + (e0 + q) * 36;
            acc += block_row(Ae, rr, x0, gmask);
            acc += block_row(Ae + 36, rr, x1, gmask);
            acc += block_row(Ae + 72, rr, x2, gmask);
            acc += block_row(Ae + 108, rr, x3, gmask);
        }
        for (; q < n; ++q) {
            const size_t e = e0 + q;
            const unsigned jj = plist[e];
            const float xj = (r < 6) ? z[6 * jj + r] : 0.f;
            acc += block_row(A + e * 36, rr, xj, gmask);
        }
        if (act) U[(size_t)nv * ld + 6 * i + r] = acc;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < nv; ++q) {
        double d = act ? (double)U[(size_t)q * ld + 6 * i + r] * (double)acc : 0.0;
        d = group_sum_d<32>(d);
        if (lane == 0) sh[q][wid] = d;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sh[threadIdx.x][w];
        part[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
        __threadfence();
    }
    if (!last_block(ticket)) return;
    for (int q = wid; q < nv; q += blockDim.x >> 5) {
        const double t = warp_sum_parts(part + (size_t)q * gridDim.x, gridDim.x);
        if (lane == 0) H[(size_t)j * (kMaxInner + 1) + q] = nrm[q] > 0.0 ? t / nrm[q] : 0.0;
    }
    if (threadIdx.x == 0) *ticket = 0;
}

// Least squares min || beta e1 - H y || by Givens rotations in FP64 (one
// thread; k <= kMaxInner).  Columns after a breakdown (zero subdiagonal or
// zero pivot) are dropped.  y is written after H's beta slot.
__device__ void inner_lsq(double* H, int k) {
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

// U_nv -= sum_{q<nv} (H[j][q] / |U_q|) U_q; |U_nv| goes to nrm[nv] and to
// H[j][nv].  With lsq_k > 0 the last block then solves the k-step least
// squares problem.
__global__ void __launch_bounds__(kInnerThreads) k_inner_orth(float* U, size_t ld, int nv, double* H,
                                                              double* nrm, int j, size_t n, double* part,
                                                              unsigned* ticket, int lsq_k) {
    __shared__ float hc[kMaxInner + 1];
    if (threadIdx.x < nv)
        hc[threadIdx.x] =
            nrm[threadIdx.x] > 0.0 ? (float)(H[(size_t)j * (kMaxInner + 1) + threadIdx.x] / nrm[threadIdx.x]) : 0.f;
    __syncthreads();
    float* w = U + (size_t)nv * ld;
    double s = 0.0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    if ((n & 3) == 0 && (ld & 3) == 0) {  // 16-byte aligned vectors (6N divisible by 4): float4 loads
        float4* w4 = reinterpret_cast<float4*>(w);
        const float4* U4 = reinterpret_cast<const float4*>(U);
        const size_t n4 = n >> 2, ld4 = ld >> 2;
        for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n4; k += stride) {
            float4 acc = w4[k];
            for (int q = 0; q < nv; ++q) {
                const float4 u = U4[(size_t)q * ld4 + k];
                const float c = -hc[q];
                acc.x = fmaf(c, u.x, acc.x);
                acc.y = fmaf(c, u.y, acc.y);
                acc.z = fmaf(c, u.z, acc.z);
                acc.w = fmaf(c, u.w, acc.w);
            }
            w4[k] = acc;
            s += (double)acc.x * acc.x;
            s += (double)acc.y * acc.y;
            s += (double)acc.z * acc.z;
            s += (double)acc.w * acc.w;
        }
    } else {
        for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += stride) {
            float acc = w[k];
            for (int q = 0; q < nv; ++q) acc = fmaf(-hc[q], U[(size_t)q * ld + k], acc);
            w[k] = acc;
            s += (double)acc * acc;
        }
    }
    block_partial(s, part);
    if (!last_block(ticket)) return;
    if (threadIdx.x < 32) {
        const double t = sqrt(warp_sum_parts(part, gridDim.x));
        if (threadIdx.x == 0) {
            nrm[nv] = t;
            H[(size_t)j * (kMaxInner + 1) + nv] = t;
            if (lsq_k > 0) inner_lsq(H, lsq_k);
            *ticket = 0;
        }
    }
}

// x = post(b, sum_i c_i Z_i): x[0:6N] = b - y, x[6N:11N] = b, x[11N:] = y.
__global__ void k_inner_post(const float* __restrict__ Z, size_t ld, int k, const double* __restrict__ c,
                             const float* b, float* x, int N) {
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    if (kk < 6 * N) {
        float acc = 0.f;
        for (int i = 0; i < k; ++i) acc += (float)c[i] * Z[(size_t)i * ld + kk];
        const float bk = b[kk];
        x[kk] = bk - acc;
        x[11 * (size_t)N + kk] = acc;
    } else if (kk < 11 * N) {
        x[kk] = b[kk];
    }
}

static int inner_alloc(fsd_handle* h) {
    LearnedState* s = learned(h);
    if (s->inner_cap >= 0) return FSD_OK;
    const size_t N = h->p.N;
    const size_t n6 = 6 * N;
    FSD_CHECK_CUDA(cudaMalloc(&s->Vi, sizeof(float) * n6 * (kMaxInner + 1)));
    FSD_CHECK_CUDA(cudaMalloc(&s->Zi, sizeof(float) * n6 * kMaxInner));
    const size_t nb = std::max<size_t>(kInnerBlocks, (8 * N + 255) / 256);
    FSD_CHECK_CUDA(cudaMalloc(&s->part, sizeof(double) * (kMaxInner + 1) * nb));
    FSD_CHECK_CUDA(cudaMalloc(&s->H, sizeof(double) * ((kMaxInner + 1) * kMaxInner + 1 + kMaxInner)));
    FSD_CHECK_CUDA(cudaMalloc(&s->nrm, sizeof(double) * (kMaxInner + 1)));
    FSD_CHECK_CUDA(cudaMalloc(&s->ticket, sizeof(unsigned)));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->ticket, 0, sizeof(unsigned), h->stream));
    s->inner_cap = kMaxInner;
    return FSD_OK;
}

bool precond_is_flexible(const fsd_handle* h) {
    return h->p.precond == FSD_PRECOND_LEARNED && h->p.learned_inner > 0 && !poly_active(h);
}

// Kernels of one inner solve on the right-hand side b into x, enqueued on st
// (for graph capture).  Basis U_j is kept unnormalised with |U_j| in nrm[j];
// each kernel applies the 1/|U_j| factors it needs.
static int inner_enqueue(fsd_handle* h, const float* b, float* x, cudaStream_t st) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    const int k = h->p.learned_inner;
    const size_t n6 = 6 * (size_t)N;
    const int rows = (8 * N + 255) / 256;
    k_inner_rhs<<<kInnerBlocks, kInnerThreads, 0, st>>>(b, s->Vi, N, s->part, s->ticket, s->H, s->nrm);
    for (int j = 0; j < k; ++j) {
        float* uj = s->Vi + (size_t)j * n6;
        float* zj = s->Zi + (size_t)j * n6;
        k_bsr_spmv_n<<<rows, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, uj, s->nrm + j, zj, N);
        k_pruned_spmv_dots<<<rows, 256, 0, st>>>(s->a_pn, s->a_plist, s->a_blocks, zj, s->Vi, n6, j + 1,
                                                 s->nrm, s->part, s->ticket, s->H, j, N);
        k_inner_orth<<<kInnerBlocks, kInnerThreads, 0, st>>>(s->Vi, n6, j + 1, s->H, s->nrm, j, n6, s->part,
                                                             s->ticket, j == k - 1 ? k : 0);
    }
    k_inner_post<<<(11 * N + 255) / 256, 256, 0, st>>>(s->Zi, n6, k, s->H + (size_t)(kMaxInner + 1) * kMaxInner + 1,
                                                       b, x, N);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

static int inner_kernels(int k) { return 2 + 3 * k; }

// (Re)capture the inner solve when the arrays it reads were reallocated or k
// changed.  The first and last kernel nodes (the only ones that touch b and
// x) are kept so that each application can point them at its own vectors.
static int inner_graph(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    const void* key[8] = {s->g_rowptr, s->g_col, s->g_val, s->a_pn, s->a_plist, s->a_blocks, s->Vi, s->Zi};
    bool same = s->gexec && s->gkey_k == h->p.learned_inner;
    for (int i = 0; i < 8 && same; ++i) same = key[i] == s->gkey[i];
    if (same) return FSD_OK;
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->gexec = nullptr;
    s->graph = nullptr;
    if (!s->cap_stream) FSD_CHECK_CUDA(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    FSD_CHECK_CUDA(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int e = inner_enqueue(h, b, x, s->cap_stream);
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
    s->node_rhs = s->node_post = nullptr;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        FSD_CHECK_CUDA(cudaGraphNodeGetType(nd, &t));
        if (t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        FSD_CHECK_CUDA(cudaGraphKernelNodeGetParams(nd, &kp));
        if (kp.func == (void*)k_inner_rhs) s->node_rhs = nd;
        if (kp.func == (void*)k_inner_post) s->node_post = nd;
    }
    if (!s->node_rhs || !s->node_post) {
        cudaGraphDestroy(g);
        return FSD_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&s->gexec, g, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        FSD_CHECK_CUDA(ie);
    }
    s->graph = g;
    for (int i = 0; i < 8; ++i) s->gkey[i] = key[i];
    s->gkey_k = h->p.learned_inner;
    s->captures += 1;
    if (getenv("FSD_DEBUG_GRAPH")) fprintf(stderr, "inner graph captured (%d)\n", s->captures);
    return FSD_OK;
}

// Point the graph's first and last kernels at b and x.
static int inner_bind(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    int N = h->p.N;
    float* u0 = s->Vi;
    double* part = s->part;
    unsigned* ticket = s->ticket;
    double* H = s->H;
    double* nrm = s->nrm;
    void* rhs_args[] = {&b, &u0, &N, &part, &ticket, &H, &nrm};
    cudaKernelNodeParams kr = {};
    kr.func = (void*)k_inner_rhs;
    kr.gridDim = dim3(kInnerBlocks);
    kr.blockDim = dim3(kInnerThreads);
    kr.kernelParams = rhs_args;
    FSD_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(s->gexec, s->node_rhs, &kr));
    const float* Z = s->Zi;
    size_t ld = 6 * (size_t)N;
    int k = h->p.learned_inner;
    const double* c = s->H + (size_t)(kMaxInner + 1) * kMaxInner + 1;
    void* post_args[] = {&Z, &ld, &k, &c, &b, &x, &N};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_inner_post;
    kp.gridDim = dim3((11 * N + 255) / 256);
    kp.blockDim = dim3(256);
    kp.kernelParams = post_args;
    FSD_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(s->gexec, s->node_post, &kp));
    return FSD_OK;
}

// x = P^-1 b.  Without inner steps G is applied once (fused with the saddle
// pre/post steps).  With k inner steps, y ~ (R_FU^pruned + D)^-1 t comes from
// k steps of GMRES on that matrix from a zero guess, right-preconditioned by
// G; the map b -> x then depends on b nonlinearly, which the flexible outer
// GMRES allows.  The inner solve is one CUDA graph launch reading b and
// writing x directly; no host synchronisation.  b and x may be the same
// vector.
int precond_apply_learned(fsd_handle* h, const float* b, float* x) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    if (poly_active(h)) return poly_apply(h, b, x);
    const int k = h->p.learned_inner;
    if (k == 0) {
        count_launch();
        k_pc_bsr<<<(8 * N + 255) / 256, 256, 0, st>>>(s->g_rowptr, s->g_col, s->g_val, b, x, N);
        FSD_CHECK_CUDA(cudaGetLastError());
        return FSD_OK;
    }
    int e = inner_graph(h, b, x);
    if (e != FSD_OK) return e;
    e = inner_bind(h, b, x);
    if (e != FSD_OK) return e;
    FSD_CHECK_CUDA(cudaGraphLaunch(s->gexec, st));
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
    const bool poly = h->p.learned_poly >= 2;
    if (poly) e = poly_alloc(h);
    else if (h->p.learned_inner > 0) e = inner_alloc(h);
    if (e != FSD_OK) return e;
    e = precond_assemble_pruned(h, pos, 1.0f, &s->a_pn, &s->a_plist, &s->a_blocks);
    if (e != FSD_OK) return e;
    if (!s->g_user) {
        e = spai_build(h);
        if (e != FSD_OK) return e;
        // The network either predicts the inner polynomial (learned_poly) or
        // corrects G on its own pattern.
        if (mpnn_loaded(h) && !poly) {
            e = mpnn_infer(h, pos, s->a_pn, s->a_plist, s->a_blocks);
            if (e != FSD_OK) return e;
        }
    }
    if (poly) {
        e = poly_prepare_products(h);
        if (e != FSD_OK) return e;
        e = poly_lambda(h);
        if (e != FSD_OK) return e;
        // Coefficients: the caller's; else the Chebyshev interval whose lower
        // end the network predicts for this configuration; else a fixed
        // interval ratio (poly_interval > 0); else a least-squares fit on
        // probe vectors.
        s->poly_ratio = -1.f;
        if (s->poly_user) {
            s->poly_source = 3;
        } else if (s->user_ratio > 0.f) {
            e = poly_set_interval(h, s->user_ratio);
            if (e != FSD_OK) return e;
            s->poly_source = 4;
        } else if (mpnn_loaded(h)) {
            double rho = 0.0;
            float log_rho = 0.f;
            e = mpnn_poly_ratio(h, pos, &rho, &log_rho);
            if (e != FSD_OK) return e;
            const bool finite = std::isfinite(log_rho);  // else the fixed interval (or 0.05)
            e = poly_set_interval(h, finite ? rho : (h->p.poly_interval > 0.f ? h->p.poly_interval : 0.05));
            if (e != FSD_OK) return e;
            s->poly_source = finite ? 1 : 4;
        } else if (h->p.poly_interval > 0.f) {
            e = poly_set_interval(h, h->p.poly_interval);
            if (e != FSD_OK) return e;
            s->poly_source = 4;
        } else {
            e = mpnn_poly_calibrate(h, h->p.learned_poly, ++s->poly_builds);
            if (e != FSD_OK) return e;
        }
    }
    h->pc_valid = true;
    return FSD_OK;
}

int learned_set_weights(fsd_handle* h, const float* host_w, int n) {
    const int e = mpnn_set_weights(h, host_w, n);
    if (e == FSD_OK) {
        learned(h)->g_user = false;
        learned(h)->poly_user = false;  // the network's coefficients from now on
        learned(h)->user_ratio = -1.f;
    }
    return e;
}

}  // namespace fsd
