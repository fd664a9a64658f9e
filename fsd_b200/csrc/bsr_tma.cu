// Block-sparse (6x6 fp32 blocks, block CSR) products of the learned
// preconditioner's inner polynomial, with the matrix streamed into shared
// memory by the Tensor Memory Accelerator.
//
// The approximate inverse G (54 MB at N = 32768, phi = 0.4) and the pruned
// lubrication matrix A are read once per product.  One CTA of 128 threads
// takes a tile of consecutive rows whose blocks (at most kTileBlocks) lie
// contiguously in memory; one thread issues a bulk copy (cp.async.bulk,
// completing on an mbarrier) of the tile's blocks into shared memory, and
// while it is in flight the threads gather the tile's row pointers and the
// operand's 6-vectors for its column indices into shared memory (every load
// issued before any is waited on).  The rows are then multiplied from shared
// memory alone, eight lanes per row.  Tiles are small so that many CTAs (up
// to ten) share an SM: the kernel is bound by the chain of L2 round trips
// per tile, which the resident tiles overlap.  The copies carry an L2
// evict-last policy, so G and A stay in L2 across the 2k - 1 products of one
// application.  Tiles are cut on the host once per preconditioner build.
//
// The mbarrier wait is bounded: when it runs out the CTA records an error
// (read by the host after the solve), waits once more (also bounded) for its
// own copy and returns without writing.
#include <algorithm>
#include <vector>

#include "fsd_device.cuh"
#include "fsd_learned.h"
#include "fsd_solver.h"

namespace fsd {

namespace {

constexpr long long kBsrSpinLimit = 1ll << 22;
__device__ int g_bsr_error = 0;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t phase) {
    for (long long n = 0; n < kBsrSpinLimit; ++n) {
        if (bar_try_wait(bar, phase)) return true;
        if (n > 32) __nanosleep(32);
    }
    return false;
}

// Bulk copy global -> this CTA's shared memory, completing on bar, with an L2
// policy: the matrices of the inner polynomial (G and A, about 75 MB at
// N = 32768, phi = 0.4) are read 2k - 1 times per application, back to back,
// and fit in the 126 MB L2 together, so their lines are marked evict-last.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(policy));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ float row6(const float* blk, int rr, float xj, unsigned gmask) {
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

}  // namespace

// Modes: 0 = first product of the Clenshaw recurrence (operand t = b[0:6N] -
// b[11N:17N], writes T = t, B = c_{k-1} t, out = c_{k-1} G t); 1 = plain
// product out = M x; 2 = last product y = G v with the saddle post step into
// xs; 3 = Clenshaw step out = c_m T + f ((2/lambda) A u - B1) - B2.
template <int MODE>
__global__ void __launch_bounds__(kBsrThreads, 8) k_bsr_tma(BsrTmaArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int sR[kTileBlocks + 1];  // the tile's row pointers, relative to its first block
    float* sG = reinterpret_cast<float*>(sm);
    float* sX = reinterpret_cast<float*>(sm + (size_t)kTileBlocks * 144);
    const int t = blockIdx.x;
    if (t >= *a.ntiles) return;  // the launch covers the tile capacity
    const int r0 = a.tile_row[t], r1 = a.tile_row[t + 1];
    const int e0 = a.rowptr[r0], e1 = a.rowptr[r1];
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t gbytes = (uint32_t)(e1 - e0) * 144u;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)), "r"(gbytes)
                     : "memory");
        if (gbytes) bulk_load(sG, a.val + (size_t)e0 * 36, gbytes, &bar);
    }
    const int N = a.N;
    const size_t offU = 11 * (size_t)N;
    // Row pointers and operand 6-vectors of the tile's columns: each thread
    // takes whole blocks, issuing every load before it waits on any.  MODE 0
    // reads the caller's saddle vector (only 4-byte alignment assumed: scalar
    // loads); the other modes read the handle's own 6N-float slots, which are
    // 8-byte aligned (float2 loads).
    {
        constexpr int kGather = (kTileBlocks + kBsrThreads - 1) / kBsrThreads;
        int rp[kGather], cj[kGather];
#pragma unroll
        for (int k = 0; k < kGather; ++k) {
            const int q = threadIdx.x + kBsrThreads * k;
            rp[k] = q <= r1 - r0 ? a.rowptr[r0 + q] : 0;
            cj[k] = q < e1 - e0 ? a.col[e0 + q] : -1;
        }
        float2 xv[kGather][3];
#pragma unroll
        for (int k = 0; k < kGather; ++k) {
            if (cj[k] < 0) continue;
            if (MODE == 0) {
                const float* x1 = a.x + 6 * (size_t)cj[k];
                const float* u1 = x1 + offU;
                xv[k][0] = make_float2(x1[0] - u1[0], x1[1] - u1[1]);
                xv[k][1] = make_float2(x1[2] - u1[2], x1[3] - u1[3]);
                xv[k][2] = make_float2(x1[4] - u1[4], x1[5] - u1[5]);
            } else {
                const float2* x2 = reinterpret_cast<const float2*>(a.x + 6 * (size_t)cj[k]);
                xv[k][0] = x2[0];
                xv[k][1] = x2[1];
                xv[k][2] = x2[2];
            }
        }
#pragma unroll
        for (int k = 0; k < kGather; ++k) {
            const int q = threadIdx.x + kBsrThreads * k;
            if (q <= r1 - r0) sR[q] = rp[k] - e0;
            if (cj[k] < 0) continue;
            float2* d2 = reinterpret_cast<float2*>(sX + 6 * (size_t)q);
            d2[0] = xv[k][0];
            d2[1] = xv[k][1];
            d2[2] = xv[k][2];
        }
    }
    const bool ok = bar_wait(&bar, 0);
    __syncthreads();  // sX and sR complete
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_bsr_error, 1);
        bar_wait(&bar, 0);  // the copy may still land in this CTA's shared memory
        return;
    }
    const int lane8 = threadIdx.x & 7;
    const int group = threadIdx.x >> 3;
    const int rr = lane8 < 6 ? lane8 : 0;
    // whole groups of eight take rows; lanes 0-5 each produce one row of the 6-vector
    for (int rl = group; rl < r1 - r0; rl += kBsrThreads / 8) {
        const int r = r0 + rl;
        const int qb = sR[rl], qe = sR[rl + 1];
        const size_t i6 = 6 * (size_t)r + lane8;
        // the row's epilogue operands, loaded before the multiply so that
        // their latency overlaps it
        float e_a = 0.f, e_b = 0.f, e_c = 0.f;
        if (lane8 < 6) {
            if (MODE == 0) {
                e_a = a.x[i6];
                e_b = a.x[offU + i6];
            } else if (MODE == 2) {
                e_a = a.b[i6];
            } else if (MODE == 3) {
                e_a = a.T[i6];
                e_b = a.B1[i6];
                e_c = a.B2 ? a.B2[i6] : 0.f;
            }
        }
        float acc = 0.f;
        for (int q = qb; q < qe; ++q) {
            const float2* g2 = reinterpret_cast<const float2*>(sG + (size_t)q * 36 + rr * 6);
            const float2* x2 = reinterpret_cast<const float2*>(sX + (size_t)q * 6);
            const float2 g01 = g2[0], g23 = g2[1], g45 = g2[2];
            const float2 x01 = x2[0], x23 = x2[1], x45 = x2[2];
            acc = fmaf(g01.x, x01.x, acc);
            acc = fmaf(g01.y, x01.y, acc);
            acc = fmaf(g23.x, x23.x, acc);
            acc = fmaf(g23.y, x23.y, acc);
            acc = fmaf(g45.x, x45.x, acc);
            acc = fmaf(g45.y, x45.y, acc);
        }
        if (MODE == 0) {
            if (lane8 < 6) {
                const float c = a.pc[a.k - 1];
                const float tv = e_a - e_b;
                a.T[i6] = tv;
                a.B[i6] = c * tv;
                a.out[i6] = c * acc;
            }
        } else if (MODE == 1) {
            if (lane8 < 6) a.out[i6] = acc;
        } else if (MODE == 2) {
            if (lane8 < 6) {
                a.xs[i6] = e_a - acc;
                a.xs[offU + i6] = acc;
            }
            if (lane8 < 5) {
                const size_t q5 = 6 * (size_t)N + 5 * (size_t)r + lane8;
                a.xs[q5] = a.b[q5];
            }
        } else {
            if (lane8 < 6) {
                const float s2 = 2.0f / a.pc[kMaxPoly];
                const float f = a.m >= 1 ? 2.0f : 1.0f;
                float v = fmaf(a.pc[a.m], e_a, f * fmaf(s2, acc, -e_b));
                if (a.B2) v -= e_c;
                a.out[i6] = v;
            }
        }
    }
}

size_t bsr_tma_smem() { return (size_t)kTileBlocks * (144 + 24); }

// Kernel entry of a mode (for launches and graph-node updates).
const void* bsr_tma_kernel(int mode) {
    switch (mode) {
        case 0: return (const void*)k_bsr_tma<0>;
        case 1: return (const void*)k_bsr_tma<1>;
        case 2: return (const void*)k_bsr_tma<2>;
        default: return (const void*)k_bsr_tma<3>;
    }
}

int bsr_tma_prepare() {
    for (int m = 0; m < 4; ++m) FSD_CHECK_CUDA(ensure_smem_limit(bsr_tma_kernel(m), bsr_tma_smem()));
    return FSD_OK;
}

void bsr_tma_launch(int mode, const BsrTmaArgs& a, int grid, cudaStream_t st) {
    const size_t smem = bsr_tma_smem();
    switch (mode) {
        case 0: k_bsr_tma<0><<<grid, kBsrThreads, smem, st>>>(a); break;
        case 1: k_bsr_tma<1><<<grid, kBsrThreads, smem, st>>>(a); break;
        case 2: k_bsr_tma<2><<<grid, kBsrThreads, smem, st>>>(a); break;
        default: k_bsr_tma<3><<<grid, kBsrThreads, smem, st>>>(a); break;
    }
}

// Pruned A (padded rows of kPrunedCap blocks) copied into block CSR.
__global__ void k_compact_pruned(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                                 const float* __restrict__ A, const int* __restrict__ rowptr, int N, int* col,
                                 float* val) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const unsigned n = pn[i];
    const int base = rowptr[i];
    for (unsigned q = 0; q < n; ++q) {
        if (lane == 0) col[base + q] = (int)plist[(size_t)i * kPrunedCap + q];
        const float* src = A + ((size_t)i * kPrunedCap + q) * 36;
        float* dst = val + (size_t)(base + q) * 36;
        for (int k = lane; k < 36; k += 32) dst[k] = src[k];
    }
}

int bsr_tma_error() {
    int e = 0;
    cudaMemcpyFromSymbol(&e, g_bsr_error, sizeof(int));
    if (e) {
        const int z = 0;
        cudaMemcpyToSymbol(g_bsr_error, &z, sizeof(int));
    }
    return e;
}

// Tiles of consecutive rows with at most kTileBlocks blocks (and rows) each,
// from a host copy of the row pointer.  Rows longer than a tile cannot occur:
// G rows hold at most kSpaiCap blocks and A rows at most kPrunedCap.
int bsr_make_tiles(const std::vector<int>& rowptr, int N, std::vector<int>& tiles) {
    tiles.clear();
    tiles.push_back(0);
    int start = 0;
    for (int r = 0; r < N; ++r) {
        if (rowptr[r + 1] - rowptr[start] > kTileBlocks || r - start >= kTileBlocks) {
            tiles.push_back(r);
            start = r;
        }
        if (rowptr[r + 1] - rowptr[r] > kTileBlocks) return FSD_ERR_BAD_PARAMS;
    }
    tiles.push_back(N);
    return FSD_OK;
}

}  // namespace fsd
