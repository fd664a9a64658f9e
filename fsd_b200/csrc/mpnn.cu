// Message-passing network for the learned block-sparse preconditioner:
// graph construction, features, forward pass, the equivariant block head,
// the approximate-inverse loss E_z ||A G z - z||^2 with its gradient,
// backward pass and Adam.  Layout and formulas: fsd_mpnn.h.
//
// The dense layers go through mp_gemm (one interface, two kernels): the
// tensor-core kernel of umma_gemm.cu with BF16 operands and FP32 accumulation,
// or an FP32 SIMT kernel used as its check.  Everything else is FP32 with
// FP64 reductions where a sum runs over the whole graph.  Every reduction has a
// fixed order, so a training run is reproducible bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fsd_brownian.h"
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_mpnn.h"
#include "fsd_profile.h"
#include "fsd_solver.h"
#include "fsd_umma.h"

namespace fsd {

namespace {
constexpr int W = kMpWidth;
constexpr int kThreads = 256;

inline int nblk(size_t n, int t = kThreads) { return (int)std::min<size_t>((n + t - 1) / t, 148 * 16); }
}  // namespace

// ------------------------------------------------------------------ graph
// Edges c -> s for the members s != c of c's two-hop set, in set order, so
// edge e of row c sits at G position sp_rowptr[c] + 1 + (e - rowptr[c]).
// rhat = (unit vector c -> s, distance); features are rotation invariants.
__device__ __forceinline__ float slog(float x) { return copysignf(log1pf(fabsf(x)), x) * 0.25f; }

__global__ void k_g_rows(const unsigned* __restrict__ sp_rowptr, int N, unsigned* rowptr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= N) rowptr[c] = sp_rowptr[c] - (unsigned)c;
}

__global__ void k_g_from_sets(const float4* __restrict__ pos, int N, Box b, const int* __restrict__ sets,
                              const unsigned* __restrict__ ns, const unsigned* __restrict__ rowptr,
                              const unsigned* __restrict__ pn, const unsigned* __restrict__ plist, ResTable tab,
                              int* src, int* dst, float4* rhat, float* x) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const float4 pc = pos[c];
    const int* S = sets + (size_t)c * kSpaiCap;
    for (unsigned a = 1; a < ns[c]; ++a) {
        const size_t e = rowptr[c] + a - 1;
        const int j = S[a];
        const float4 pj = pos[j];
        const float3 r = min_image_rn(make_float3(pj.x - pc.x, pj.y - pc.y, pj.z - pc.z), b);
        const float d = sqrtf(dist2_rn(r));
        src[e] = c;
        dst[e] = j;
        rhat[e] = make_float4(r.x / d, r.y / d, r.z / d, d);
        bool direct = false;
        for (unsigned q = 0; q < pn[c]; ++q)
            if ((int)plist[(size_t)c * kPrunedCap + q] == j) direct = true;
        const float h = d - 2.0f;
        float cf[10];
        res_interp<10>(tab, d, 0, cf);
        float* o = x + e * kMpFeat;
        o[0] = logf(fmaxf(h, 1e-4f)) * 0.2f;
        o[1] = h;
        o[2] = expf(-10.0f * fmaxf(h, 0.0f));
        o[3] = 2.0f / d;
#pragma unroll
        for (int k = 0; k < 10; ++k) o[4 + k] = slog(cf[k]);
        o[14] = direct ? 1.0f : 0.0f;
        o[15] = 1.0f;
    }
}

// rev[e] = position of the opposite edge j -> i (or -1 if absent).
__global__ void k_g_rev(const unsigned* __restrict__ rowptr, const int* __restrict__ src, const int* __restrict__ dst,
                        int E, int* rev) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int i = src[e], j = dst[e];
    int r = -1;
    for (unsigned f = rowptr[j]; f < rowptr[j + 1]; ++f)
        if (dst[f] == i) {
            r = (int)f;
            break;
        }
    rev[e] = r;
}

// J_i = (A_ii)^-1 for the self block of the pruned matrix (FP64 Gauss-Jordan
// on an SPD 6x6 block), and the row's degree in the G graph.
__global__ void k_g_jinv(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                         const float* __restrict__ A, int N, float* J) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int s = 0;
    for (unsigned q = 0; q < pn[i]; ++q)
        if (plist[(size_t)i * kPrunedCap + q] == (unsigned)i) s = (int)q;
    const float* a = A + ((size_t)i * kPrunedCap + s) * 36;
    double m[6][12];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 12; ++c) m[r][c] = (c < 6) ? (double)a[r * 6 + c] : (c - 6 == r ? 1.0 : 0.0);
    for (int c = 0; c < 6; ++c) {
        int p = c;
        for (int r = c + 1; r < 6; ++r)
            if (fabs(m[r][c]) > fabs(m[p][c])) p = r;
        if (p != c)
            for (int q = 0; q < 12; ++q) {
                const double t = m[c][q];
                m[c][q] = m[p][q];
                m[p][q] = t;
            }
        const double piv = m[c][c];
        const double inv = piv != 0.0 ? 1.0 / piv : 0.0;
        for (int q = 0; q < 12; ++q) m[c][q] *= inv;
        for (int r = 0; r < 6; ++r)
            if (r != c) {
                const double f = m[r][c];
                for (int q = 0; q < 12; ++q) m[r][q] -= f * m[c][q];
            }
    }
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) J[(size_t)i * 36 + r * 6 + c] = (float)m[r][6 + c];
}

// ------------------------------------------------------------ SIMT GEMM
// Y[r][o] = act(sum_k X(r,k) W[o][k] + b[o]) (+ R[r][o]), with X a row-wise
// concatenation of up to three 64-wide (or one 16-wide) parts, each part read
// through an optional row index.  64 rows x 64 outputs per block, 4x4 per thread.
struct GemmIn {
    const float* p[3];
    const int* idx[3];
    int width;   // columns per part (64, or 16 for the input layer)
    int parts;
};

__global__ void __launch_bounds__(256) k_gemm_simt(GemmIn in, int rows, const float* __restrict__ Wt, int O,
                                                   const float* __restrict__ bias, int relu,
                                                   const float* __restrict__ resid, float* __restrict__ Y,
                                                   int ldy) {
    __shared__ float xs[16][65];
    __shared__ float ws[16][65];
    const int K = in.width * in.parts;
    const int r0 = blockIdx.x * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int kk = t & 15, rr = t >> 4;
            const int k = k0 + kk;
            const int part = k / in.width, col = k - part * in.width;
            const int r = r0 + rr;
            float v = 0.f;
            if (r < rows) {
                const int src = in.idx[part] ? in.idx[part][r] : r;
                v = in.p[part][(size_t)src * in.width + col];
            }
            xs[kk][rr] = v;
            ws[kk][rr] = (rr < O) ? Wt[(size_t)rr * K + k] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float xv[4], wv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) xv[a] = xs[kk][ty * 4 + a];
#pragma unroll
            for (int c = 0; c < 4; ++c) wv[c] = ws[kk][tx * 4 + c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] += xv[a] * wv[c];
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int r = r0 + ty * 4 + a;
        if (r >= rows) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int o = tx * 4 + c;
            if (o >= O) continue;
            float v = acc[a][c] + bias[o];
            if (relu) v = fmaxf(v, 0.f);
            if (resid) v += resid[(size_t)r * ldy + o];
            Y[(size_t)r * ldy + o] = v;
        }
    }
}

// dX[r][k] = sum_o dY[r][o] W[o][k]   (dX dense, K columns)
__global__ void __launch_bounds__(256) k_gemm_dx_simt(const float* __restrict__ dY, int rows, int O,
                                                      const float* __restrict__ Wt, int K, float* __restrict__ dX) {
    __shared__ float ds[16][65];
    __shared__ float ws[16][65];
    const int r0 = blockIdx.x * 64, k0b = blockIdx.y * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    for (int o0 = 0; o0 < O; o0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int oo = t & 15, rr = t >> 4;
            const int o = o0 + oo, r = r0 + rr, k = k0b + rr;
            ds[oo][rr] = (r < rows && o < O) ? dY[(size_t)r * O + o] : 0.f;
            ws[oo][rr] = (k < K && o < O) ? Wt[(size_t)o * K + k] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int oo = 0; oo < 16; ++oo) {
            float dv[4], wv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) dv[a] = ds[oo][ty * 4 + a];
#pragma unroll
            for (int c = 0; c < 4; ++c) wv[c] = ws[oo][tx * 4 + c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] += dv[a] * wv[c];
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int r = r0 + ty * 4 + a;
        if (r >= rows) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = k0b + tx * 4 + c;
            if (k < K) dX[(size_t)r * K + k] = acc[a][c];
        }
    }
}

// Partial weight gradients: part[blk][o][k] = sum over the block's rows of
// dY[r][o] X(r,k), and part[blk][o][K] = sum dY[r][o] (bias).  One block per
// kRowsPerPart rows; a second kernel sums the partials in block order.
constexpr int kRowsPerPart = 512;

__global__ void __launch_bounds__(256) k_gemm_dw_part(GemmIn in, int rows, const float* __restrict__ dY, int O,
                                                      float* __restrict__ part) {
    const int K = in.width * in.parts;
    const int r0 = blockIdx.x * kRowsPerPart;
    const int r1 = min(rows, r0 + kRowsPerPart);
    const int KK = K + 1;
    float* out = part + (size_t)blockIdx.x * O * KK;
    for (int t = threadIdx.x; t < O * KK; t += blockDim.x) {
        const int o = t / KK, k = t - o * KK;
        float s = 0.f;
        if (k < K) {
            const int p = k / in.width, col = k - p * in.width;
            for (int r = r0; r < r1; ++r) {
                const int src = in.idx[p] ? in.idx[p][r] : r;
                s += dY[(size_t)r * O + o] * in.p[p][(size_t)src * in.width + col];
            }
        } else {
            for (int r = r0; r < r1; ++r) s += dY[(size_t)r * O + o];
        }
        out[t] = s;
    }
}

// dW[o][k] += sum_blk part, db[o] += sum_blk part[..][K].
__global__ void k_gemm_dw_reduce(const float* __restrict__ part, int nparts, int O, int K, float* dW, float* db) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int KK = K + 1;
    if (t >= O * KK) return;
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += part[(size_t)b * O * KK + t];
    const int o = t / KK, k = t - o * KK;
    if (k < K) dW[(size_t)o * K + k] += (float)s;
    else db[o] += (float)s;
}

// ----------------------------------------------------------- aggregation
// out[i] = mean over row i's edges of in[e] (64 wide).  One warp per row, two
// columns per lane.
__global__ void k_seg_mean(const unsigned* __restrict__ rowptr, const float* __restrict__ in, int N, float* out) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const unsigned b = rowptr[i], e = rowptr[i + 1];
    float s0 = 0.f, s1 = 0.f;
    for (unsigned f = b; f < e; ++f) {
        s0 += in[(size_t)f * W + lane];
        s1 += in[(size_t)f * W + 32 + lane];
    }
    const float inv = e > b ? 1.0f / (float)(e - b) : 0.f;
    out[(size_t)i * W + lane] = s0 * inv;
    out[(size_t)i * W + 32 + lane] = s1 * inv;
}

// d(in)[e] (+)= d(out)[src(e)] / deg(src(e))
__global__ void k_seg_mean_bwd(const unsigned* __restrict__ rowptr, const float* __restrict__ dout, int N,
                               float* din, int accumulate) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const unsigned b = rowptr[i], e = rowptr[i + 1];
    const float inv = e > b ? 1.0f / (float)(e - b) : 0.f;
    const float g0 = dout[(size_t)i * W + lane] * inv, g1 = dout[(size_t)i * W + 32 + lane] * inv;
    for (unsigned f = b; f < e; ++f) {
        if (accumulate) {
            din[(size_t)f * W + lane] += g0;
            din[(size_t)f * W + 32 + lane] += g1;
        } else {
            din[(size_t)f * W + lane] = g0;
            din[(size_t)f * W + 32 + lane] = g1;
        }
    }
}

// Node gradients from a gathered-edge input gradient dX (E x ldx), parts at
// column offsets cs (gathered by src) and cd (gathered by dst):
// dh[i] += sum_{e in row i} dX[e][cs + :] + dX[rev(e)][cd + :].
__global__ void k_node_from_edges(const unsigned* __restrict__ rowptr, const int* __restrict__ rev,
                                  const float* __restrict__ dX, int ldx, int cs, int cd, int N, float* dh) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    float s0 = 0.f, s1 = 0.f;
    for (unsigned f = rowptr[i]; f < rowptr[i + 1]; ++f) {
        s0 += dX[(size_t)f * ldx + cs + lane];
        s1 += dX[(size_t)f * ldx + cs + 32 + lane];
        const int r = rev[f];
        if (r >= 0) {
            s0 += dX[(size_t)r * ldx + cd + lane];
            s1 += dX[(size_t)r * ldx + cd + 32 + lane];
        }
    }
    dh[(size_t)i * W + lane] += s0;
    dh[(size_t)i * W + 32 + lane] += s1;
}

// y[r][c] = x[r][coff + c] * (mask[r][c] > 0) for a 64-wide slice (ReLU backward
// through a stored post-activation), optionally accumulated.
__global__ void k_relu_bwd(const float* __restrict__ g, int ldg, int goff, const float* __restrict__ act, size_t rows,
                           float* __restrict__ out) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= rows * W) return;
    const size_t r = t / W;
    const int c = (int)(t - r * W);
    out[t] = act[t] > 0.f ? g[r * ldg + goff + c] : 0.f;
}

__global__ void k_add_slice(const float* __restrict__ g, int ldg, int goff, size_t rows, float* __restrict__ out) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= rows * W) return;
    const size_t r = t / W;
    out[t] += g[r * ldg + goff + (int)(t - r * W)];
}

// ------------------------------------------------------------------ head
__device__ __forceinline__ void axis_block(const float* o, float3 r, float* B) {
    // B(o, r): [o0 rr + o1 (I - rr), o2 [r]x ; o3 [r]x, o4 rr + o5 (I - rr)]
    const float rv[3] = {r.x, r.y, r.z};
    // [r]x v = r x v:  rows (0, -rz, ry), (rz, 0, -rx), (-ry, rx, 0)
    const float cx[3][3] = {{0.f, -r.z, r.y}, {r.z, 0.f, -r.x}, {-r.y, r.x, 0.f}};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const float rr = rv[a] * rv[b];
            const float id = (a == b) ? 1.f : 0.f;
            B[a * 6 + b] = o[0] * rr + o[1] * (id - rr);
            B[a * 6 + 3 + b] = o[2] * cx[a][b];
            B[(3 + a) * 6 + b] = o[3] * cx[a][b];
            B[(3 + a) * 6 + 3 + b] = o[4] * rr + o[5] * (id - rr);
        }
}

// <dB, dB/do_k> for the six basis tensors of axis_block.
__device__ __forceinline__ void axis_block_grad(const float* dB, float3 r, float* go) {
    const float rv[3] = {r.x, r.y, r.z};
    const float cx[3][3] = {{0.f, -r.z, r.y}, {r.z, 0.f, -r.x}, {-r.y, r.x, 0.f}};
    float g[6] = {};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const float rr = rv[a] * rv[b];
            const float id = (a == b) ? 1.f : 0.f;
            g[0] += dB[a * 6 + b] * rr;
            g[1] += dB[a * 6 + b] * (id - rr);
            g[2] += dB[a * 6 + 3 + b] * cx[a][b];
            g[3] += dB[(3 + a) * 6 + b] * cx[a][b];
            g[4] += dB[(3 + a) * 6 + 3 + b] * rr;
            g[5] += dB[(3 + a) * 6 + 3 + b] * (id - rr);
        }
    for (int k = 0; k < 6; ++k) go[k] = g[k];
}

// Correction added to G (block CSR of the two-hop sets; row i = [self,
// edges of i]).  One thread per row.
__global__ void k_head_blocks(const unsigned* __restrict__ rowptr, const float4* __restrict__ rhat,
                              const float* __restrict__ oe, const float* __restrict__ on, const float* __restrict__ J,
                              int N, float* G) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const unsigned b = rowptr[i], e = rowptr[i + 1];
    const size_t base = (size_t)b + i;
    float Ji[36];
    for (int k = 0; k < 36; ++k) Ji[k] = J[(size_t)i * 36 + k];
    float S[36];
    for (int k = 0; k < 36; ++k) S[k] = 0.f;
    const float ct = on[(size_t)i * kMpHeadN + 0], cr = on[(size_t)i * kMpHeadN + 1];
    for (int d = 0; d < 6; ++d) S[d * 7] = (d < 3 ? ct : cr);
    float B[36];
    for (unsigned f = b; f < e; ++f) {
        const float4 rh = rhat[f];
        const float3 r = make_float3(rh.x, rh.y, rh.z);
        axis_block(oe + (size_t)f * kMpHeadE + 6, r, B);
        for (int k = 0; k < 36; ++k) S[k] += B[k];
        axis_block(oe + (size_t)f * kMpHeadE, r, B);
        float* out = G + (base + 1 + (f - b)) * 36;
        for (int a = 0; a < 6; ++a)
            for (int c = 0; c < 6; ++c) {
                float s = 0.f;
                for (int q = 0; q < 6; ++q) s += Ji[a * 6 + q] * B[q * 6 + c];
                out[a * 6 + c] += s;
            }
    }
    float* out = G + base * 36;
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c < 6; ++c) {
            float s = 0.f;
            for (int q = 0; q < 6; ++q) s += Ji[a * 6 + q] * S[q * 6 + c];
            out[a * 6 + c] += s;
        }
}

// From dG (block CSR like G) to head gradients: dB = J_i^T dG.
__global__ void k_head_bwd(const unsigned* __restrict__ rowptr, const float4* __restrict__ rhat,
                           const float* __restrict__ J, const float* __restrict__ dG, int N, float* doe, float* don) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const unsigned b = rowptr[i], e = rowptr[i + 1];
    const int base = (int)b + i;
    float Ji[36];
    for (int k = 0; k < 36; ++k) Ji[k] = J[(size_t)i * 36 + k];
    float dS[36];
    {
        const float* g = dG + (size_t)base * 36;
        for (int a = 0; a < 6; ++a)
            for (int c = 0; c < 6; ++c) {
                float s = 0.f;
                for (int q = 0; q < 6; ++q) s += Ji[q * 6 + a] * g[q * 6 + c];
                dS[a * 6 + c] = s;
            }
    }
    don[(size_t)i * kMpHeadN + 0] = dS[0] + dS[7] + dS[14];
    don[(size_t)i * kMpHeadN + 1] = dS[21] + dS[28] + dS[35];
    for (int k = 2; k < kMpHeadN; ++k) don[(size_t)i * kMpHeadN + k] = 0.f;
    float dB[36], go[6];
    for (unsigned f = b; f < e; ++f) {
        const float4 rh = rhat[f];
        const float3 r = make_float3(rh.x, rh.y, rh.z);
        const float* g = dG + (size_t)(base + 1 + (f - b)) * 36;
        for (int a = 0; a < 6; ++a)
            for (int c = 0; c < 6; ++c) {
                float s = 0.f;
                for (int q = 0; q < 6; ++q) s += Ji[q * 6 + a] * g[q * 6 + c];
                dB[a * 6 + c] = s;
            }
        float* d = doe + (size_t)f * kMpHeadE;
        axis_block_grad(dB, r, go);
        for (int k = 0; k < 6; ++k) d[k] = go[k];
        axis_block_grad(dS, r, go);
        for (int k = 0; k < 6; ++k) d[6 + k] = go[k];
        for (int k = 12; k < kMpHeadE; ++k) d[k] = 0.f;
    }
}

// ------------------------------------------------------------------ loss
// u = G Z for P probe columns stored probe-major (P x 6N).
__global__ void k_bsr_multi(const int* __restrict__ rowptr, const int* __restrict__ col, const float* __restrict__ G,
                            const float* __restrict__ Z, float* __restrict__ U, int N, int P) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 3, r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const size_t n6 = 6 * (size_t)N;
    for (int p = 0; p < P; ++p) {
        float acc = 0.f;
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const int j = col[e];
            const float xj = (r < 6) ? Z[p * n6 + 6 * j + r] : 0.f;
            const float* Ge = G + (size_t)e * 36 + (r < 6 ? r : 0) * 6;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const float xc = __shfl_sync(gmask, xj, c, 8);
                if (r < 6) acc += Ge[c] * xc;
            }
        }
        if (r < 6) U[p * n6 + 6 * i + r] = acc;
    }
}

__global__ void k_pruned_multi(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                               const float* __restrict__ A, const float* __restrict__ X, float* __restrict__ Y, int N,
                               int P) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 3, r = threadIdx.x & 7;
    if (i >= N) return;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const size_t n6 = 6 * (size_t)N;
    for (int p = 0; p < P; ++p) {
        float acc = 0.f;
        for (unsigned s = 0; s < pn[i]; ++s) {
            const size_t e = (size_t)i * kPrunedCap + s;
            const unsigned j = plist[e];
            const float xj = (r < 6) ? X[p * n6 + 6 * j + r] : 0.f;
            const float* Ae = A + e * 36 + (r < 6 ? r : 0) * 6;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const float xc = __shfl_sync(gmask, xj, c, 8);
                if (r < 6) acc += Ae[c] * xc;
            }
        }
        if (r < 6) Y[p * n6 + 6 * i + r] = acc;
    }
}

// R = (V - Z) * scale in place of V; part[b] = partial sum (V - Z)^2.
__global__ void __launch_bounds__(kThreads) k_resid(float* V, const float* __restrict__ Z, size_t n, float scale,
                                                    double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const float d = V[k] - Z[k];
        s += (double)d * d;
        V[k] = d * scale;
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

__global__ void k_sum_part(const double* part, int nb, double scale, double* out) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) s += part[b];
    s = group_sum_d<32>(s);
    if (threadIdx.x == 0) *out = s * scale;
}

// dG block (i, col e) = sum_p dU_p[i] Z_p[j]^T.
__global__ void k_dG(const int* __restrict__ rowptr, const int* __restrict__ col, const float* __restrict__ dU,
                     const float* __restrict__ Z, int N, int P, float* dG) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const size_t n6 = 6 * (size_t)N;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
        const int j = col[e];
        float g[36] = {};
        for (int p = 0; p < P; ++p) {
            const float* du = dU + p * n6 + 6 * (size_t)i;
            const float* z = Z + p * n6 + 6 * (size_t)j;
            for (int a = 0; a < 6; ++a)
                for (int c = 0; c < 6; ++c) g[a * 6 + c] += du[a] * z[c];
        }
        float* out = dG + (size_t)e * 36;
        for (int k = 0; k < 36; ++k) out[k] = g[k];
    }
}

// ------------------------------------------------------------------ Adam
__global__ void k_adam(float* w, const float* __restrict__ g, float* m, float* v, int n, float lr, float b1, float b2,
                       float c1, float c2, float eps, float clip) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float gk = g[k];
    gk = fminf(fmaxf(gk, -clip), clip);
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// ------------------------------------------------------------ host side
struct MpState {
    int N = 0;
    int E = 0, E_cap = 0;
    float rg = 0.f;
    unsigned* cnt = nullptr;     // N+1 (scan output)
    unsigned* scan = nullptr;
    int* src = nullptr;
    int* dst = nullptr;
    int* rev = nullptr;
    float4* rhat = nullptr;
    float* x = nullptr;          // E x 16
    float* J = nullptr;          // N x 36
    // activations
    float* e[kMpLayers + 1] = {};
    float* m[kMpLayers] = {};
    float* h[kMpLayers + 1] = {};
    float* a[kMpLayers] = {};
    float* u[kMpLayers] = {};    // relu(W_h [h, a] + b) per layer
    float* oe = nullptr;         // E x 16
    float* on = nullptr;         // N x 16
    // backward
    float* dX = nullptr;         // E x 192
    float* dXn = nullptr;        // N x 128
    float* de = nullptr;         // E x 64
    float* dm = nullptr;         // E x 64
    float* dh = nullptr;         // N x 64
    float* dh2 = nullptr;        // N x 64
    float* dA = nullptr;         // N x 64
    float* du = nullptr;         // N x 64
    float* doe = nullptr;
    float* don = nullptr;
    float* dG = nullptr;
    float* dwpart = nullptr;
    size_t dwpart_cap = 0;
    // weights
    float* w = nullptr;
    float* gw = nullptr;
    float* mw = nullptr;
    float* vw = nullptr;
    bool loaded = false;
    int adam_t = 0;
    // probes
    float* Zp = nullptr;
    float* Up = nullptr;
    float* Vp = nullptr;
    int P_cap = 0;
    double* part = nullptr;
    double* loss = nullptr;
    // inner-polynomial training: Chebyshev basis images W_m = AG T_m(S) t
    // (k x P x 6N), three recurrence slots (3 x P x 6N), Gram partials
    float* pw = nullptr;
    float* pb = nullptr;
    size_t pw_cap = 0, pb_cap = 0;
    double* gpart = nullptr;
    size_t gpart_cap = 0;
    bool use_umma = true;
    std::vector<unsigned> h_cnt;
};

static MpState* mp(fsd_handle* h) {
    LearnedState* s = learned(h);
    if (!s->mp) s->mp = new MpState();
    return (MpState*)s->mp;
}

template <class T> static int grow(T** p, size_t n) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    FSD_CHECK_CUDA(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1)));
    return FSD_OK;
}

#define MP_TRY(x)                   \
    do {                            \
        int s_ = (x);               \
        if (s_ != FSD_OK) return s_; \
    } while (0)

void mpnn_free(fsd_handle* h) {
    LearnedState* ls = (LearnedState*)h->learned;
    if (!ls || !ls->mp) return;
    MpState* s = (MpState*)ls->mp;
    void* ptrs[] = {s->cnt, s->scan, s->src, s->dst, s->rev, s->rhat, s->x, s->J, s->oe, s->on, s->dX, s->dXn, s->de,
                    s->dm, s->dh, s->dh2, s->dA, s->du, s->doe, s->don, s->dG, s->dwpart, s->w, s->gw, s->mw, s->vw,
                    s->Zp, s->Up, s->Vp, s->part, s->loss, s->pw, s->pb, s->gpart};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int l = 0; l <= kMpLayers; ++l) {
        if (s->e[l]) cudaFree(s->e[l]);
        if (s->h[l]) cudaFree(s->h[l]);
    }
    for (int l = 0; l < kMpLayers; ++l) {
        if (s->m[l]) cudaFree(s->m[l]);
        if (s->a[l]) cudaFree(s->a[l]);
        if (s->u[l]) cudaFree(s->u[l]);
    }
    delete s;
    ls->mp = nullptr;
}

static int mp_alloc_static(fsd_handle* h) {
    MpState* s = mp(h);
    if (s->N) return FSD_OK;
    const int N = h->p.N;
    s->N = N;
    MP_TRY(grow(&s->cnt, N + 1));
    MP_TRY(grow(&s->scan, scan_scratch_elems(N)));
    MP_TRY(grow(&s->J, (size_t)N * 36));
    for (int l = 0; l <= kMpLayers; ++l) MP_TRY(grow(&s->h[l], (size_t)N * W));
    for (int l = 0; l < kMpLayers; ++l) {
        MP_TRY(grow(&s->a[l], (size_t)N * W));
        MP_TRY(grow(&s->u[l], (size_t)N * W));
    }
    MP_TRY(grow(&s->on, (size_t)N * kMpHeadN));
    MP_TRY(grow(&s->w, MpLayout::total));
    MP_TRY(grow(&s->gw, MpLayout::total));
    MP_TRY(grow(&s->mw, MpLayout::total));
    MP_TRY(grow(&s->vw, MpLayout::total));
    MP_TRY(grow(&s->part, 4096));
    MP_TRY(grow(&s->loss, 4));
    s->h_cnt.resize(1);
    return FSD_OK;
}

static int mp_alloc_edges(fsd_handle* h, int E) {
    MpState* s = mp(h);
    if (E <= s->E_cap) return FSD_OK;
    const int cap = E + E / 8 + 1024;
    MP_TRY(grow(&s->src, cap));
    MP_TRY(grow(&s->dst, cap));
    MP_TRY(grow(&s->rev, cap));
    MP_TRY(grow(&s->rhat, cap));
    MP_TRY(grow(&s->x, (size_t)cap * kMpFeat));
    for (int l = 0; l <= kMpLayers; ++l) MP_TRY(grow(&s->e[l], (size_t)cap * W));
    for (int l = 0; l < kMpLayers; ++l) MP_TRY(grow(&s->m[l], (size_t)cap * W));
    MP_TRY(grow(&s->oe, (size_t)cap * kMpHeadE));
    s->E_cap = cap;
    // backward buffers are grown on first use (training only)
    if (s->dX) {
        cudaFree(s->dX);
        s->dX = nullptr;
    }
    return FSD_OK;
}

static int mp_alloc_backward(fsd_handle* h) {
    MpState* s = mp(h);
    if (s->dX) return FSD_OK;
    const int N = s->N;
    const size_t cap = s->E_cap;
    MP_TRY(grow(&s->dX, cap * 3 * W));
    MP_TRY(grow(&s->dXn, (size_t)N * 2 * W));
    MP_TRY(grow(&s->de, cap * W));
    MP_TRY(grow(&s->dm, cap * W));
    MP_TRY(grow(&s->dh, (size_t)N * W));
    MP_TRY(grow(&s->dh2, (size_t)N * W));
    MP_TRY(grow(&s->dA, (size_t)N * W));
    MP_TRY(grow(&s->du, (size_t)N * W));
    MP_TRY(grow(&s->doe, cap * kMpHeadE));
    MP_TRY(grow(&s->don, (size_t)N * kMpHeadN));
    MP_TRY(grow(&s->dG, (cap + N) * 36));
    return FSD_OK;
}

// Dense layer through the tensor-core kernel (BF16 operands, FP32
// accumulation) or the FP32 SIMT kernel.
static void mp_gemm(fsd_handle* h, const GemmIn& in, int rows, const float* Wt, int O, const float* b, int relu,
                    const float* resid, float* Y) {
    MpState* s = mp(h);
    if (rows <= 0) return;
    count_launch();
    if (s->use_umma && umma_gemm_supported(in.width * in.parts, O)) {
        umma_gemm(in.p, in.idx, in.width, in.parts, rows, Wt, O, b, relu, resid, Y, h->stream);
        return;
    }
    k_gemm_simt<<<(rows + 63) / 64, 256, 0, h->stream>>>(in, rows, Wt, O, b, relu, resid, Y, O);
}

static void mp_gemm_dx(fsd_handle* h, const float* dY, int rows, int O, const float* Wt, int K, float* dX) {
    MpState* s = mp(h);
    if (rows <= 0) return;
    count_launch();
    if (s->use_umma && umma_gemm_dx_supported(O, K)) {
        umma_gemm_dx(dY, rows, O, Wt, K, dX, h->stream);
        return;
    }
    dim3 g((rows + 63) / 64, (K + 63) / 64);
    k_gemm_dx_simt<<<g, 256, 0, h->stream>>>(dY, rows, O, Wt, K, dX);
}

static int mp_gemm_dw(fsd_handle* h, const GemmIn& in, int rows, const float* dY, int O, float* dW, float* db) {
    MpState* s = mp(h);
    if (rows <= 0) return FSD_OK;
    const int K = in.width * in.parts;
    if (s->use_umma && umma_gemm_dw_supported(K, O)) {
        const size_t need = umma_dw_part_floats(rows, K, O);
        if (need > s->dwpart_cap) {
            MP_TRY(grow(&s->dwpart, need));
            s->dwpart_cap = need;
        }
        for (int i = 0; i < 4; ++i) count_launch();
        umma_gemm_dw(in.p, in.idx, in.width, in.parts, rows, dY, O, dW, db, s->dwpart, h->stream);
        return FSD_OK;
    }
    const int nparts = (rows + kRowsPerPart - 1) / kRowsPerPart;
    const size_t need = (size_t)nparts * O * (K + 1);
    if (need > s->dwpart_cap) {
        MP_TRY(grow(&s->dwpart, need));
        s->dwpart_cap = need;
    }
    count_launch();
    k_gemm_dw_part<<<nparts, 256, 0, h->stream>>>(in, rows, dY, O, s->dwpart);
    count_launch();
    k_gemm_dw_reduce<<<(O * (K + 1) + 255) / 256, 256, 0, h->stream>>>(s->dwpart, nparts, O, K, dW, db);
    return FSD_OK;
}

static GemmIn cat3(const float* e, const float* hs, const float* hd, const int* src, const int* dst) {
    GemmIn g{};
    g.p[0] = e;
    g.p[1] = hs;
    g.p[2] = hd;
    g.idx[0] = nullptr;
    g.idx[1] = src;
    g.idx[2] = dst;
    g.width = W;
    g.parts = 3;
    return g;
}
static GemmIn cat2(const float* a, const float* b) {
    GemmIn g{};
    g.p[0] = a;
    g.p[1] = b;
    g.width = W;
    g.parts = 2;
    return g;
}
static GemmIn one(const float* a, int width) {
    GemmIn g{};
    g.p[0] = a;
    g.width = width;
    g.parts = 1;
    return g;
}

// Graph (the two-hop sets of the approximate inverse), features and J for
// these positions; spai_build must have run for them.
static int mp_graph(fsd_handle* h, const float4* pos, const unsigned* a_pn, const unsigned* a_plist,
                    const float* a_blocks) {
    MP_TRY(mp_alloc_static(h));
    MpState* s = mp(h);
    LearnedState* ls = learned(h);
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    const int E = ls->g_nnzb - N;
    MP_TRY(mp_alloc_edges(h, E));
    s->E = E;
    count_launch();
    k_g_rows<<<(N + 1 + 127) / 128, 128, 0, st>>>(ls->sp_rowptr, N, s->cnt);
    count_launch();
    k_g_from_sets<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, ls->sp_sets, ls->sp_size, s->cnt, a_pn, a_plist,
                                                   ResTable{h->d_res_dist, h->d_res_vals}, s->src, s->dst, s->rhat,
                                                   s->x);
    if (E) {
        count_launch();
        k_g_rev<<<(E + 255) / 256, 256, 0, st>>>(s->cnt, s->src, s->dst, E, s->rev);
    }
    count_launch();
    k_g_jinv<<<(N + 127) / 128, 128, 0, st>>>(a_pn, a_plist, a_blocks, N, s->J);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

static int mp_forward(fsd_handle* h) {
    MpState* s = mp(h);
    const int N = s->N, E = s->E;
    cudaStream_t st = h->stream;
    const float* w = s->w;
    mp_gemm(h, one(s->x, kMpFeat), E, w + MpLayout::W_in, W, w + MpLayout::b_in, 1, nullptr, s->e[0]);
    count_launch();
    k_seg_mean<<<(N * 32 + 255) / 256, 256, 0, st>>>(s->cnt, s->e[0], N, s->h[0]);
    for (int l = 0; l < kMpLayers; ++l) {
        const float* L = w + MpLayout::layer(l);
        mp_gemm(h, cat3(s->e[l], s->h[l], s->h[l], s->src, s->dst), E, L + MpLayout::W_m, W, L + MpLayout::b_m, 1,
                nullptr, s->m[l]);
        // e[l+1] = e[l] + m[l]
        FSD_CHECK_CUDA(cudaMemcpyAsync(s->e[l + 1], s->e[l], sizeof(float) * (size_t)E * W, cudaMemcpyDeviceToDevice,
                                       st));
        count_launch();
        k_add_slice<<<(unsigned)(((size_t)E * W + 255) / 256), 256, 0, st>>>(s->m[l], W, 0, E, s->e[l + 1]);
        count_launch();
        k_seg_mean<<<(N * 32 + 255) / 256, 256, 0, st>>>(s->cnt, s->m[l], N, s->a[l]);
        mp_gemm(h, cat2(s->h[l], s->a[l]), N, L + MpLayout::W_h, W, L + MpLayout::b_h, 1, nullptr, s->u[l]);
        FSD_CHECK_CUDA(cudaMemcpyAsync(s->h[l + 1], s->h[l], sizeof(float) * (size_t)N * W, cudaMemcpyDeviceToDevice,
                                       st));
        count_launch();
        k_add_slice<<<(unsigned)(((size_t)N * W + 255) / 256), 256, 0, st>>>(s->u[l], W, 0, N, s->h[l + 1]);
    }
    mp_gemm(h, cat3(s->e[kMpLayers], s->h[kMpLayers], s->h[kMpLayers], s->src, s->dst), E, w + MpLayout::W_o,
            kMpHeadE, w + MpLayout::b_o, 0, nullptr, s->oe);
    mp_gemm(h, one(s->h[kMpLayers], W), N, w + MpLayout::W_n, kMpHeadN, w + MpLayout::b_n, 0, nullptr, s->on);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Add the network's correction to the approximate inverse in place.
static int mp_head(fsd_handle* h) {
    MpState* s = mp(h);
    LearnedState* ls = learned(h);
    const int N = s->N;
    count_launch();
    k_head_blocks<<<(N + 127) / 128, 128, 0, h->stream>>>(s->cnt, s->rhat, s->oe, s->on, s->J, N, ls->g_val);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Backward from d(oe), d(on) to the weight gradient s->gw (accumulated).
static int mp_backward(fsd_handle* h) {
    MpState* s = mp(h);
    const int N = s->N, E = s->E;
    cudaStream_t st = h->stream;
    const float* w = s->w;
    float* gw = s->gw;
    const size_t EW = (size_t)E * W, NW = (size_t)N * W;
    const unsigned ge = (unsigned)((EW + 255) / 256), gn = (unsigned)((NW + 255) / 256);
    // heads
    MP_TRY(mp_gemm_dw(h, one(s->h[kMpLayers], W), N, s->don, kMpHeadN, gw + MpLayout::W_n, gw + MpLayout::b_n));
    mp_gemm_dx(h, s->don, N, kMpHeadN, w + MpLayout::W_n, W, s->dh);  // dh = d h3 (node head)
    MP_TRY(mp_gemm_dw(h, cat3(s->e[kMpLayers], s->h[kMpLayers], s->h[kMpLayers], s->src, s->dst), E, s->doe, kMpHeadE,
                      gw + MpLayout::W_o, gw + MpLayout::b_o));
    mp_gemm_dx(h, s->doe, E, kMpHeadE, w + MpLayout::W_o, 3 * W, s->dX);
    // de = dX[:, 0:64]; dh += gathered parts
    FSD_CHECK_CUDA(cudaMemsetAsync(s->de, 0, sizeof(float) * EW, st));
    count_launch();
    k_add_slice<<<ge, 256, 0, st>>>(s->dX, 3 * W, 0, E, s->de);
    count_launch();
    k_node_from_edges<<<(N * 32 + 255) / 256, 256, 0, st>>>(s->cnt, s->rev, s->dX, 3 * W, W, 2 * W, N, s->dh);
    for (int l = kMpLayers - 1; l >= 0; --l) {
        const float* L = w + MpLayout::layer(l);
        float* GL = gw + MpLayout::layer(l);
        // h[l+1] = h[l] + u[l], u = relu(W_h [h[l], a[l]] + b_h)
        count_launch();
        k_relu_bwd<<<gn, 256, 0, st>>>(s->dh, W, 0, s->u[l], N, s->du);
        MP_TRY(mp_gemm_dw(h, cat2(s->h[l], s->a[l]), N, s->du, W, GL + MpLayout::W_h, GL + MpLayout::b_h));
        mp_gemm_dx(h, s->du, N, W, L + MpLayout::W_h, 2 * W, s->dXn);
        // d h[l] = dh (residual) + dXn[:, 0:64];  d a[l] = dXn[:, 64:128]
        count_launch();
        k_add_slice<<<gn, 256, 0, st>>>(s->dXn, 2 * W, 0, N, s->dh);
        // a = seg_mean(m): dm = d a / deg scattered to edges;  e[l+1] = e[l] + m: dm += de
        FSD_CHECK_CUDA(cudaMemcpy2DAsync(s->dA, sizeof(float) * W, s->dXn + W, sizeof(float) * 2 * W,
                                         sizeof(float) * W, N, cudaMemcpyDeviceToDevice, st));
        count_launch();
        k_seg_mean_bwd<<<(N * 32 + 255) / 256, 256, 0, st>>>(s->cnt, s->dA, N, s->dm, 0);
        count_launch();
        k_add_slice<<<ge, 256, 0, st>>>(s->de, W, 0, E, s->dm);
        // m = relu(W_m [e[l], h[l]_src, h[l]_dst] + b_m)
        count_launch();
        k_relu_bwd<<<ge, 256, 0, st>>>(s->dm, W, 0, s->m[l], E, s->dm);
        MP_TRY(mp_gemm_dw(h, cat3(s->e[l], s->h[l], s->h[l], s->src, s->dst), E, s->dm, W, GL + MpLayout::W_m,
                          GL + MpLayout::b_m));
        mp_gemm_dx(h, s->dm, E, W, L + MpLayout::W_m, 3 * W, s->dX);
        // d e[l] = de (residual) + dX[:, 0:64];  d h[l] += gathered
        count_launch();
        k_add_slice<<<ge, 256, 0, st>>>(s->dX, 3 * W, 0, E, s->de);
        count_launch();
        k_node_from_edges<<<(N * 32 + 255) / 256, 256, 0, st>>>(s->cnt, s->rev, s->dX, 3 * W, W, 2 * W, N, s->dh);
    }
    // h[0] = seg_mean(e[0]): de += scatter(dh / deg)
    count_launch();
    k_seg_mean_bwd<<<(N * 32 + 255) / 256, 256, 0, st>>>(s->cnt, s->dh, N, s->de, 1);
    // e[0] = relu(W_in x + b_in)
    count_launch();
    k_relu_bwd<<<ge, 256, 0, st>>>(s->de, W, 0, s->e[0], E, s->dm);
    MP_TRY(mp_gemm_dw(h, one(s->x, kMpFeat), E, s->dm, W, gw + MpLayout::W_in, gw + MpLayout::b_in));
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Loss L = sum_p ||A G z_p - z_p||^2 / (P 6N) for the probes z in s->Zp and,
// when grad, the gradient dL/dG_ij = sum_p (A dR_p)[i] z_p[j]^T (A symmetric),
// then through the head.
static int mp_loss(fsd_handle* h, int P, bool grad) {
    MpState* s = mp(h);
    LearnedState* ls = learned(h);
    const int N = s->N;
    cudaStream_t st = h->stream;
    const size_t n = (size_t)P * 6 * N;
    const int rows = (8 * N + 255) / 256;
    count_launch();
    k_bsr_multi<<<rows, 256, 0, st>>>(ls->g_rowptr, ls->g_col, ls->g_val, s->Zp, s->Up, N, P);
    count_launch();
    k_pruned_multi<<<rows, 256, 0, st>>>(ls->a_pn, ls->a_plist, ls->a_blocks, s->Up, s->Vp, N, P);
    const double inv = 1.0 / ((double)P * 6.0 * N);
    count_launch();
    k_resid<<<296, kThreads, 0, st>>>(s->Vp, s->Zp, n, (float)(2.0 * inv), s->part);
    count_launch();
    k_sum_part<<<1, 32, 0, st>>>(s->part, 296, inv, s->loss);
    if (!grad) return FSD_OK;
    count_launch();
    k_pruned_multi<<<rows, 256, 0, st>>>(ls->a_pn, ls->a_plist, ls->a_blocks, s->Vp, s->Up, N, P);
    count_launch();
    k_dG<<<(N + 127) / 128, 128, 0, st>>>(ls->g_rowptr, ls->g_col, s->Up, s->Zp, N, P, s->dG);
    count_launch();
    k_head_bwd<<<(N + 127) / 128, 128, 0, st>>>(s->cnt, s->rhat, s->J, s->dG, N, s->doe, s->don);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// z = w - A G0 w: the residual one application of the approximate inverse
// leaves, probes for the correction's loss (the approximate inverse itself
// is optimal for white-noise probes on its pattern).
__global__ void k_sub(const float* __restrict__ a, float* __restrict__ b, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        b[k] = a[k] - b[k];
}

static int mp_probes(fsd_handle* h, int P) {
    MpState* s = mp(h);
    if (P > s->P_cap) {
        const size_t n = (size_t)P * 6 * s->N;
        MP_TRY(grow(&s->Zp, n));
        MP_TRY(grow(&s->Up, n));
        MP_TRY(grow(&s->Vp, n));
        s->P_cap = P;
    }
    return FSD_OK;
}

// ------------------------------------------------------------ entry points
int mpnn_set_weights(fsd_handle* h, const float* host_w, int n) {
    if (n != MpLayout::total) return FSD_ERR_BAD_PARAMS;
    MP_TRY(mp_alloc_static(h));
    MpState* s = mp(h);
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->w, host_w, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->mw, 0, sizeof(float) * n, h->stream));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->vw, 0, sizeof(float) * n, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    s->adam_t = 0;
    s->loaded = true;
    return FSD_OK;
}

int mpnn_get_weights(fsd_handle* h, float* host_w, int n) {
    MpState* s = mp(h);
    if (n != MpLayout::total || !s->loaded) return FSD_ERR_BAD_PARAMS;
    FSD_CHECK_CUDA(cudaMemcpyAsync(host_w, s->w, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return FSD_OK;
}

// Weights with the Adam moments and step count, so that training can move
// between handles (one per box size) without restarting the optimiser.
int mpnn_get_state(fsd_handle* h, float* host, int n, int* t) {
    MpState* s = mp(h);
    if (n != 3 * MpLayout::total || !s->loaded) return FSD_ERR_BAD_PARAMS;
    const size_t m = MpLayout::total;
    FSD_CHECK_CUDA(cudaMemcpyAsync(host, s->w, sizeof(float) * m, cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaMemcpyAsync(host + m, s->mw, sizeof(float) * m, cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaMemcpyAsync(host + 2 * m, s->vw, sizeof(float) * m, cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    *t = s->adam_t;
    return FSD_OK;
}

int mpnn_set_state(fsd_handle* h, const float* host, int n, int t) {
    if (n != 3 * MpLayout::total || t < 0) return FSD_ERR_BAD_PARAMS;
    MP_TRY(mpnn_set_weights(h, host, MpLayout::total));
    MpState* s = mp(h);
    const size_t m = MpLayout::total;
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->mw, host + m, sizeof(float) * m, cudaMemcpyHostToDevice, h->stream));
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->vw, host + 2 * m, sizeof(float) * m, cudaMemcpyHostToDevice, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    s->adam_t = t;
    return FSD_OK;
}

bool mpnn_loaded(fsd_handle* h) {
    LearnedState* ls = (LearnedState*)h->learned;
    return ls && ls->mp && ((MpState*)ls->mp)->loaded;
}

void mpnn_use_umma(fsd_handle* h, bool on) { mp(h)->use_umma = on; }

// Inference: graph, forward, head -> correction added to the approximate
// inverse (precond_build of FSD_PRECOND_LEARNED, after spai_build).  With
// the tensor-core layers, a commit wait that ran out is reported here.
int mpnn_infer(fsd_handle* h, const float4* pos, const unsigned* a_pn, const unsigned* a_plist,
               const float* a_blocks) {
    MP_TRY(mp_graph(h, pos, a_pn, a_plist, a_blocks));
    MP_TRY(mp_forward(h));
    MP_TRY(mp_head(h));
    if (mp(h)->use_umma) {
        FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
        if (umma_error() != 0) return FSD_ERR_DEVICE_WAIT;
    }
    return FSD_OK;
}

// Loss and gradient for given probes z (host P x 6N), or for z = w - A G0 w
// with w standard normals drawn from (seed, step); with lr > 0 also one Adam
// step.  The neighbour
// list must be current for pos; the pruned matrix is assembled here.
int mpnn_train_step(fsd_handle* h, const float4* pos, const float* host_probes, int P, uint32_t step, float lr,
                    float* loss_out, float* host_grad) {
    LearnedState* ls = learned(h);
    if (!mpnn_loaded(h) || P < 1) return FSD_ERR_BAD_PARAMS;
    MpState* s = mp(h);
    MP_TRY(precond_assemble_pruned(h, pos, 1.0f, &ls->a_pn, &ls->a_plist, &ls->a_blocks));
    MP_TRY(spai_build(h));
    MP_TRY(mp_probes(h, P));
    const size_t n = (size_t)P * 6 * s->N;
    if (host_probes) {
        FSD_CHECK_CUDA(cudaMemcpyAsync(s->Zp, host_probes, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    } else {
        const int rows = (8 * s->N + 255) / 256;
        gaussian(h, s->Vp, n, step, kStreamLearned, 1.0f);
        count_launch();
        k_bsr_multi<<<rows, 256, 0, h->stream>>>(ls->g_rowptr, ls->g_col, ls->g_val, s->Vp, s->Up, s->N, P);
        count_launch();
        k_pruned_multi<<<rows, 256, 0, h->stream>>>(ls->a_pn, ls->a_plist, ls->a_blocks, s->Up, s->Zp, s->N, P);
        count_launch();
        k_sub<<<296, kThreads, 0, h->stream>>>(s->Vp, s->Zp, n);
    }
    MP_TRY(mpnn_infer(h, pos, ls->a_pn, ls->a_plist, ls->a_blocks));
    MP_TRY(mp_alloc_backward(h));
    MP_TRY(mp_loss(h, P, true));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->gw, 0, sizeof(float) * MpLayout::total, h->stream));
    MP_TRY(mp_backward(h));
    if (lr > 0.f) {
        s->adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)s->adam_t), c2 = 1.f - powf(b2, (float)s->adam_t);
        count_launch();
        k_adam<<<(MpLayout::total + 255) / 256, 256, 0, h->stream>>>(s->w, s->gw, s->mw, s->vw, MpLayout::total, lr,
                                                                     b1, b2, c1, c2, 1e-8f, 1.0f);
    }
    double loss = 0.0;
    FSD_CHECK_CUDA(cudaMemcpyAsync(&loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (host_grad)
        FSD_CHECK_CUDA(cudaMemcpyAsync(host_grad, s->gw, sizeof(float) * MpLayout::total, cudaMemcpyDeviceToHost,
                                       h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (s->use_umma && umma_error() != 0) return FSD_ERR_DEVICE_WAIT;
    if (loss_out) *loss_out = (float)loss;
    return FSD_OK;
}

// ---------------------------------------------------- learned inner polynomial
// The network's use in the polynomial inner solve (poly.cu): the Chebyshev
// coefficients of q for a configuration are the means over particles of the
// node head's first k outputs.  Training minimises, for probe vectors t,
//   L(c) = E_t ||t - AG q_c(AG) t||^2 / ||t||^2 = E_t (t.t - 2 c.g + c^T M c) / t.t
// with W_m = AG T_m(S) t, g_m = W_m . t, M_ml = W_m . W_l: W and the Gram
// entries are formed on the device, dL/dc on the host, and dL/dc / N is fed
// to every particle's node head output for the network's backward pass.

// pc[m] = mean_i on[i][m] for m < k (one warp per m, fixed order).
__global__ void k_poly_pool(const float* __restrict__ on, int N, int k, float* pc) {
    const int m = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (m >= k) return;
    double sum = 0.0;
    for (int i = lane; i < N; i += 32) sum += on[(size_t)i * kMpHeadN + m];
    sum = group_sum_d<32>(sum);
    if (lane == 0) pc[m] = (float)(sum / N);
}

// out = f ((2/lambda) W - Bm) - Bprev (Bprev may be null): the Chebyshev step
// T_{m+1}(S) t = 2 S T_m(S) t - T_{m-1}(S) t with S = (2/lambda) AG - I.
__global__ void k_cheb_next(const float* __restrict__ Wm, const float* __restrict__ Bm,
                            const float* __restrict__ Bprev, size_t n, const float* __restrict__ pc, float f,
                            float* __restrict__ out) {
    const float s2 = 2.0f / pc[kMaxPoly];
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        float v = f * fmaf(s2, Wm[q], -Bm[q]);
        if (Bprev) v -= Bprev[q];
        out[q] = v;
    }
}

constexpr int kGramChunk = 128;
constexpr int kGramBlocks = 32;

// Partial dot products of the k + 1 vectors (t_p, W_0p .. W_{k-1}p) of probe
// p = blockIdx.y: pair q = (a <= b) in row-major order of the upper triangle;
// part[(p * npairs + q) * gridDim.x + blockIdx.x].
__global__ void __launch_bounds__(256) k_poly_gram(const float* __restrict__ T, const float* __restrict__ Wb, int k,
                                                   int P, size_t n6, double* part) {
    __shared__ float xs[kMaxPoly + 1][kGramChunk];
    const int p = blockIdx.y;
    const int nvec = k + 1, npairs = nvec * (nvec + 1) / 2;
    int a = -1, b = -1;
    if ((int)threadIdx.x < npairs) {
        int q = threadIdx.x;
        for (int r = 0; r < nvec; ++r) {
            if (q < nvec - r) {
                a = r;
                b = r + q;
                break;
            }
            q -= nvec - r;
        }
    }
    double acc = 0.0;
    for (size_t c0 = (size_t)blockIdx.x * kGramChunk; c0 < n6; c0 += (size_t)gridDim.x * kGramChunk) {
        __syncthreads();
        for (int idx = threadIdx.x; idx < nvec * kGramChunk; idx += blockDim.x) {
            const int v = idx / kGramChunk, e = idx % kGramChunk;
            const size_t g = c0 + e;
            float val = 0.f;
            if (g < n6) val = v == 0 ? T[(size_t)p * n6 + g] : Wb[((size_t)(v - 1) * P + p) * n6 + g];
            xs[v][e] = val;
        }
        __syncthreads();
        if (a >= 0)
            for (int e = 0; e < kGramChunk; ++e) acc += (double)xs[a][e] * (double)xs[b][e];
    }
    if (a >= 0) part[((size_t)p * npairs + threadIdx.x) * gridDim.x + blockIdx.x] = acc;
}

struct PolyGrad {
    float g[kMpHeadN];
};

// dL/d on[i][m] = g[m] for every particle i.
__global__ void k_fill_don(float* don, int N, PolyGrad pg) {
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q < (size_t)N * kMpHeadN) don[q] = pg.g[q % kMpHeadN];
}

int mpnn_poly_coeffs(fsd_handle* h, const float4* pos, float* pc, int k) {
    LearnedState* ls = learned(h);
    MP_TRY(mp_graph(h, pos, ls->a_pn, ls->a_plist, ls->a_blocks));
    MP_TRY(mp_forward(h));
    MpState* s = mp(h);
    count_launch();
    k_poly_pool<<<1, 32 * kMaxPoly, 0, h->stream>>>(s->on, s->N, k, pc);
    FSD_CHECK_CUDA(cudaGetLastError());
    if (s->use_umma) {
        FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
        if (umma_error() != 0) return FSD_ERR_DEVICE_WAIT;
    }
    return FSD_OK;
}

// Small dense solve M c = g (partial pivoting, FP64); false if singular.
static bool solve_small(std::vector<double> M, std::vector<double> g, int k, std::vector<double>& c) {
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int r = col + 1; r < k; ++r)
            if (std::fabs(M[r * k + col]) > std::fabs(M[piv * k + col])) piv = r;
        if (!(std::fabs(M[piv * k + col]) > 0.0)) return false;
        if (piv != col) {
            for (int q = 0; q < k; ++q) std::swap(M[col * k + q], M[piv * k + q]);
            std::swap(g[col], g[piv]);
        }
        for (int r = col + 1; r < k; ++r) {
            const double f = M[r * k + col] / M[col * k + col];
            for (int q = col; q < k; ++q) M[r * k + q] -= f * M[col * k + q];
            g[r] -= f * g[col];
        }
    }
    c.assign(k, 0.0);
    for (int r = k - 1; r >= 0; --r) {
        double v = g[r];
        for (int q = r + 1; q < k; ++q) v -= M[r * k + q] * c[q];
        c[r] = v / M[r * k + r];
    }
    return true;
}

// Gram entries of P probe vectors t_p drawn from (seed, step) for the
// current G, A and spectral bound: tt = t.t, g_m = W_m . t, M_ml = W_m . W_l
// with W_m = AG T_m(S) t (S = (2/lambda) AG - I), m, l < k.
struct PolyGram {
    double tt = 0.0;
    std::vector<double> g, M;
};

static int poly_gram(fsd_handle* h, int P, uint32_t step, int k, std::vector<PolyGram>& out) {
    LearnedState* ls = learned(h);
    MpState* s = mp(h);
    cudaStream_t st = h->stream;
    MP_TRY(mp_alloc_static(h));
    MP_TRY(mp_probes(h, P));
    const int N = s->N;
    const size_t n6 = 6 * (size_t)N, nP = (size_t)P * n6;
    if ((size_t)k * nP > s->pw_cap) {
        MP_TRY(grow(&s->pw, (size_t)k * nP));
        s->pw_cap = (size_t)k * nP;
    }
    if (3 * nP > s->pb_cap) {
        MP_TRY(grow(&s->pb, 3 * nP));
        s->pb_cap = 3 * nP;
    }
    const int nvec = k + 1, npairs = nvec * (nvec + 1) / 2;
    const size_t ngp = (size_t)P * npairs * kGramBlocks;
    if (ngp > s->gpart_cap) {
        MP_TRY(grow(&s->gpart, ngp));
        s->gpart_cap = ngp;
    }
    gaussian(h, s->Zp, nP, step, kStreamLearned, 1.0f);
    const int rows = (8 * N + 255) / 256;
    const float* Bprev = nullptr;
    const float* Bm = s->Zp;
    for (int m = 0; m < k; ++m) {
        float* Wm = s->pw + (size_t)m * nP;
        count_launch();
        k_bsr_multi<<<rows, 256, 0, st>>>(ls->g_rowptr, ls->g_col, ls->g_val, Bm, s->Up, N, P);
        count_launch();
        k_pruned_multi<<<rows, 256, 0, st>>>(ls->a_pn, ls->a_plist, ls->a_blocks, s->Up, Wm, N, P);
        if (m + 1 < k) {
            float* o = s->pb + (size_t)(m % 3) * nP;
            count_launch();
            k_cheb_next<<<nblk(nP), kThreads, 0, st>>>(Wm, Bm, Bprev, nP, ls->pc, m == 0 ? 1.0f : 2.0f, o);
            Bprev = Bm;
            Bm = o;
        }
    }
    count_launch();
    k_poly_gram<<<dim3(kGramBlocks, P), 256, 0, st>>>(s->Zp, s->pw, k, P, n6, s->gpart);
    FSD_CHECK_CUDA(cudaGetLastError());
    std::vector<double> part(ngp);
    FSD_CHECK_CUDA(cudaMemcpyAsync(part.data(), s->gpart, sizeof(double) * ngp, cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    auto pair_index = [&](int a, int b) {
        if (a > b) std::swap(a, b);
        return a * nvec - a * (a - 1) / 2 + (b - a);
    };
    out.assign(P, PolyGram());
    for (int p = 0; p < P; ++p) {
        auto entry = [&](int a, int b) {
            const double* q = part.data() + ((size_t)p * npairs + pair_index(a, b)) * kGramBlocks;
            double v = 0.0;
            for (int blk = 0; blk < kGramBlocks; ++blk) v += q[blk];
            return v;
        };
        PolyGram& G = out[p];
        G.tt = entry(0, 0);
        G.g.resize(k);
        G.M.resize((size_t)k * k);
        for (int m = 0; m < k; ++m) {
            G.g[m] = entry(0, 1 + m);
            for (int l = 0; l < k; ++l) G.M[(size_t)m * k + l] = entry(1 + m, 1 + l);
        }
    }
    return FSD_OK;
}

// Mean relative residual E ||t - W c||^2 / ||t||^2 over probes [p0, p1).
static double poly_loss(const std::vector<PolyGram>& gr, int p0, int p1, const std::vector<double>& c) {
    const int k = (int)c.size();
    double loss = 0.0;
    for (int p = p0; p < p1; ++p) {
        double cMc = 0.0, cg = 0.0;
        for (int m = 0; m < k; ++m) {
            cg += c[m] * gr[p].g[m];
            for (int l = 0; l < k; ++l) cMc += c[m] * gr[p].M[(size_t)m * k + l] * c[l];
        }
        loss += (gr[p].tt - 2.0 * cg + cMc) / gr[p].tt;
    }
    return loss / (p1 - p0);
}

// Least-squares coefficients over probes [p0, p1); false if singular.
static bool poly_fit(const std::vector<PolyGram>& gr, int p0, int p1, int k, std::vector<double>& c) {
    std::vector<double> Ms((size_t)k * k, 0.0), gs(k, 0.0);
    for (int p = p0; p < p1; ++p)
        for (int m = 0; m < k; ++m) {
            gs[m] += gr[p].g[m] / gr[p].tt;
            for (int l = 0; l < k; ++l) Ms[(size_t)m * k + l] += gr[p].M[(size_t)m * k + l] / gr[p].tt;
        }
    return solve_small(Ms, gs, k, c);
}

// Least-squares fit of the coefficients to four probe vectors drawn at this
// build (the learned_poly form without a network and without a fixed
// interval); its loss is recorded in the learned state.
int mpnn_poly_calibrate(fsd_handle* h, int k, uint32_t step) {
    LearnedState* ls = learned(h);
    ls->poly_loss_net = -1.f;
    std::vector<PolyGram> gr;
    MP_TRY(poly_gram(h, 4, step, k, gr));
    std::vector<double> cfit;
    if (!poly_fit(gr, 0, 4, k, cfit)) return FSD_ERR_BREAKDOWN;
    ls->poly_loss_fit = (float)poly_loss(gr, 0, 4, cfit);
    float c[kMaxPoly] = {};
    for (int m = 0; m < k; ++m) c[m] = (float)cfit[m];
    FSD_CHECK_CUDA(cudaMemcpyAsync(ls->pc, c, sizeof(float) * kMaxPoly, cudaMemcpyHostToDevice, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    ls->poly_source = 2;
    return FSD_OK;
}

int mpnn_poly_train_step(fsd_handle* h, const float4* pos, int P, uint32_t step, float lr, int k, int natural,
                         float* loss_out, float* loss_opt_out, float* host_grad, float* host_coef,
                         float* host_coef_opt) {
    LearnedState* ls = learned(h);
    if (!mpnn_loaded(h) || P < 1 || k < 2 || k > kMaxPoly) return FSD_ERR_BAD_PARAMS;
    MpState* s = mp(h);
    cudaStream_t st = h->stream;
    MP_TRY(poly_alloc(h));
    MP_TRY(precond_assemble_pruned(h, pos, 1.0f, &ls->a_pn, &ls->a_plist, &ls->a_blocks));
    MP_TRY(spai_build(h));
    MP_TRY(poly_lambda(h));
    MP_TRY(mpnn_poly_coeffs(h, pos, ls->pc, k));
    std::vector<float> c32(kMaxPoly + 1);
    FSD_CHECK_CUDA(cudaMemcpyAsync(c32.data(), ls->pc, sizeof(float) * (kMaxPoly + 1), cudaMemcpyDeviceToHost, st));
    std::vector<PolyGram> gr;
    MP_TRY(poly_gram(h, P, step, k, gr));
    const int N = s->N;
    std::vector<double> c(k), grad(k, 0.0);
    for (int m = 0; m < k; ++m) c[m] = c32[m];
    const double loss = poly_loss(gr, 0, P, c);
    for (int p = 0; p < P; ++p)
        for (int m = 0; m < k; ++m) {
            double Mc = 0.0;
            for (int l = 0; l < k; ++l) Mc += gr[p].M[(size_t)m * k + l] * c[l];
            grad[m] += 2.0 * (Mc - gr[p].g[m]) / (gr[p].tt * P);
        }
    std::vector<double> copt;
    double loss_opt = -1.0;
    if (poly_fit(gr, 0, P, k, copt)) loss_opt = poly_loss(gr, 0, P, copt);
    // The loss is quadratic in c with Hessian 2 Mbar (Mbar = mean_p M_p / tt_p),
    // badly conditioned in the Chebyshev coefficients.  With `natural` the
    // network is fed the Gauss-Newton direction Mbar^-1 dL/dc = 2 (c - c_opt)
    // instead of dL/dc.
    if (natural && !copt.empty())
        for (int m = 0; m < k; ++m) grad[m] = 2.0 * (c[m] - copt[m]);
    // backward: the node head's outputs each carry the gradient / N
    MP_TRY(mp_alloc_backward(h));
    PolyGrad pg{};
    for (int m = 0; m < k; ++m) pg.g[m] = (float)(grad[m] / N);
    count_launch();
    k_fill_don<<<(unsigned)(((size_t)N * kMpHeadN + 255) / 256), 256, 0, st>>>(s->don, N, pg);
    FSD_CHECK_CUDA(cudaMemsetAsync(s->doe, 0, sizeof(float) * (size_t)s->E_cap * kMpHeadE, st));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->gw, 0, sizeof(float) * MpLayout::total, st));
    MP_TRY(mp_backward(h));
    if (lr > 0.f) {
        s->adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)s->adam_t), c2 = 1.f - powf(b2, (float)s->adam_t);
        count_launch();
        k_adam<<<(MpLayout::total + 255) / 256, 256, 0, st>>>(s->w, s->gw, s->mw, s->vw, MpLayout::total, lr, b1, b2,
                                                             c1, c2, 1e-8f, 1.0f);
    }
    if (host_grad)
        FSD_CHECK_CUDA(cudaMemcpyAsync(host_grad, s->gw, sizeof(float) * MpLayout::total, cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    if (s->use_umma && umma_error() != 0) return FSD_ERR_DEVICE_WAIT;
    if (loss_out) *loss_out = (float)loss;
    if (loss_opt_out) *loss_opt_out = (float)loss_opt;
    for (int m = 0; m < k; ++m) {
        if (host_coef) host_coef[m] = (float)c[m];
        if (host_coef_opt) host_coef_opt[m] = copt.empty() ? 0.f : (float)copt[m];
    }
    return FSD_OK;
}

// ------------------------------------------- learned Chebyshev interval
// The network's use in the default learned_poly mode: it predicts, for a
// configuration, the lower end a = rho lambda of the Chebyshev interval of
// the inner polynomial, log rho being the mean over particles of the node
// head's first output.  It is trained on the interval ratio that gave the
// fewest outer GMRES iterations in solves of the solver's own configurations
// (a squared error in log rho, one scalar per configuration).
constexpr double kRatioMin = 1e-3, kRatioMax = 0.5;

int mpnn_poly_ratio(fsd_handle* h, const float4* pos, double* rho, float* log_rho) {
    LearnedState* ls = learned(h);
    MP_TRY(poly_alloc(h));
    MP_TRY(mpnn_poly_coeffs(h, pos, ls->pc, 1));  // pc[0] = mean of the first node output (synchronised)
    float s0 = 0.f;
    FSD_CHECK_CUDA(cudaMemcpyAsync(&s0, ls->pc, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (log_rho) *log_rho = s0;
    *rho = std::min(kRatioMax, std::max(kRatioMin, std::exp((double)s0)));
    return FSD_OK;
}

int mpnn_ratio_train_step(fsd_handle* h, const float4* pos, float target_log_rho, float lr, float* loss,
                          float* pred_log_rho, float* host_grad) {
    LearnedState* ls = learned(h);
    if (!mpnn_loaded(h)) return FSD_ERR_BAD_PARAMS;
    MpState* s = mp(h);
    cudaStream_t st = h->stream;
    MP_TRY(precond_assemble_pruned(h, pos, 1.0f, &ls->a_pn, &ls->a_plist, &ls->a_blocks));
    MP_TRY(spai_build(h));
    double rho = 0.0;
    float s0 = 0.f;
    MP_TRY(mpnn_poly_ratio(h, pos, &rho, &s0));
    const double d = (double)s0 - (double)target_log_rho;
    if (!std::isfinite(d)) {  // e.g. overlapping particles: no gradient, no update
        if (loss) *loss = (float)d;
        if (pred_log_rho) *pred_log_rho = s0;
        return FSD_ERR_BREAKDOWN;
    }
    MP_TRY(mp_alloc_backward(h));
    PolyGrad pg{};
    pg.g[0] = (float)(2.0 * d / s->N);  // d(d^2)/d s0, spread over the particles' outputs
    count_launch();
    k_fill_don<<<(unsigned)(((size_t)s->N * kMpHeadN + 255) / 256), 256, 0, st>>>(s->don, s->N, pg);
    FSD_CHECK_CUDA(cudaMemsetAsync(s->doe, 0, sizeof(float) * (size_t)s->E_cap * kMpHeadE, st));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->gw, 0, sizeof(float) * MpLayout::total, st));
    MP_TRY(mp_backward(h));
    if (lr > 0.f) {
        s->adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)s->adam_t), c2 = 1.f - powf(b2, (float)s->adam_t);
        count_launch();
        k_adam<<<(MpLayout::total + 255) / 256, 256, 0, st>>>(s->w, s->gw, s->mw, s->vw, MpLayout::total, lr, b1, b2,
                                                             c1, c2, 1e-8f, 1.0f);
    }
    if (host_grad)
        FSD_CHECK_CUDA(cudaMemcpyAsync(host_grad, s->gw, sizeof(float) * MpLayout::total, cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    if (s->use_umma && umma_error() != 0) return FSD_ERR_DEVICE_WAIT;
    if (loss) *loss = (float)(d * d);
    if (pred_log_rho) *pred_log_rho = s0;
    return FSD_OK;
}

}  // namespace fsd
