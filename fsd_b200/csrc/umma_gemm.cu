// Dense layers of the message-passing network on the 5th-generation tensor
// cores: tcgen05.mma kind::f16 with BF16 operands from shared memory and the
// FP32 accumulator in tensor memory (TMEM), read back with tcgen05.ld.
//
// One CTA (128 threads, four warps) computes a 128-row tile:
//   forward  Y[128 x O]  = X[128 x K] W^T      (M = 128, N = O, K = 16..192)
//   backward dX[128 x K] = dY[128 x O] W       (M = 128, N = K, K-dim = O)
// Threads stage both operands as BF16 in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, stored so that core matrices
// adjacent along K are LBO bytes apart and 8-row groups SBO bytes apart.
// One elected thread issues the K/16 MMAs and commits them to an mbarrier;
// all threads wait on it (bounded: a wait that runs out sets an error flag,
// waits once more, frees TMEM and skips the epilogue) and then each warp
// loads its 32 TMEM lanes (rows) for the epilogue.
#include <cuda_bf16.h>
#include <cstdint>

#include "fsd_internal.h"
#include "fsd_umma.h"

namespace fsd {

namespace {
constexpr int kRows = 128;
constexpr int kThreads = 128;
constexpr long long kSpinLimit = 1ll << 24;

__device__ int g_umma_error = 0;  // set when an mbarrier wait ran out (read by umma_error())

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (K-major, no swizzle, sm_100 version 1).
__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, N, M.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with `rows`
// rows: core matrix (row / 8, k / 8) at ((k/8) * rows/8 + row/8) * 128 bytes,
// 16 bytes per row inside it.  So LBO = rows/8 * 128 and SBO = 128.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int rows) {
    return (uint32_t)(((k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    for (long long n = 0; n < kSpinLimit; ++n) {
        if (mbar_try_wait(bar, phase)) return true;
        if (n > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, int ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__host__ __device__ constexpr int tmem_cols(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 256)); }

struct Parts {
    const float* p[3];
    const int* idx[3];
};

// Common MMA driver: A (kRows x Kd) and B (Nn x Kd) are staged; issue Kd/16
// MMAs into TMEM and wait.  Returns false if the wait ran out.
__device__ bool run_mma(unsigned char* sa, unsigned char* sb, int Kd, int Nn, uint32_t tmem, uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    fence_after();
    if (threadIdx.x == 0) {
        const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
        const uint32_t lbo_a = (kRows / 8) * 128, lbo_b = (uint32_t)(Nn / 8) * 128;
        const uint32_t idesc = make_idesc(kRows, Nn);
        for (int ks = 0; ks < Kd / 16; ++ks) {
            const uint64_t da = make_desc(a0 + (uint32_t)ks * 2 * lbo_a, lbo_a, 128);
            const uint64_t db = make_desc(b0 + (uint32_t)ks * 2 * lbo_b, lbo_b, 128);
            mma_bf16(tmem, da, db, idesc, ks > 0);
        }
        mma_commit(bar);
    }
    bool ok = mbar_wait(bar, 0);
    if (!ok) {
        atomicExch(&g_umma_error, 1);
        mbar_wait(bar, 0);  // give the MMAs in flight a second bounded chance before TMEM is freed
    }
    // tcgen05.ld is warp-collective: every thread takes the same branch.
    ok = __syncthreads_and(ok) != 0;
    fence_after();
    return ok;
}
}  // namespace

// Forward dense layer.  Dynamic shared memory: A tile kRows x K and B tile O x K (BF16).
__global__ void __launch_bounds__(kThreads) k_umma_fwd(Parts in, int width, int parts, int rows,
                                                       const float* __restrict__ Wt, int O,
                                                       const float* __restrict__ bias, int relu,
                                                       const float* __restrict__ resid, float* __restrict__ Y) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int K = width * parts;
    unsigned char* sa = smem;
    unsigned char* sb = smem + (size_t)kRows * K * 2;
    const int r0 = blockIdx.x * kRows;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) tmem_alloc(&tmem_base, tmem_cols(O));
    if (threadIdx.x == 0) mbar_init(&bar);
    // A: row r of the tile, all K columns (gathered parts), converted to BF16
    for (int t = threadIdx.x; t < kRows * K; t += blockDim.x) {
        const int rr = t / K, k = t - rr * K;
        const int part = k / width, col = k - part * width;
        const int r = r0 + rr;
        float v = 0.f;
        if (r < rows) {
            const int src = in.idx[part] ? in.idx[part][r] : r;
            v = in.p[part][(size_t)src * width + col];
        }
        st_bf16(sa, kmajor_off(rr, k, kRows), v);
    }
    for (int t = threadIdx.x; t < O * K; t += blockDim.x) {
        const int o = t / K, k = t - o * K;
        st_bf16(sb, kmajor_off(o, k, O), Wt[(size_t)o * K + k]);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    const bool ok = run_mma(sa, sb, K, O, tmem, &bar);
    if (ok) {
        const int row = warp * 32 + (threadIdx.x & 31);
        const int r = r0 + row;
        for (int c0 = 0; c0 < O; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (r < rows) {
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int o = c0 + c;
                    float y = v[c] + bias[o];
                    if (relu) y = fmaxf(y, 0.f);
                    if (resid) y += resid[(size_t)r * O + o];
                    Y[(size_t)r * O + o] = y;
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(O));
}

// Backward dense layer dX = dY W.  A = dY tile (kRows x O), B = W^T (K x O).
__global__ void __launch_bounds__(kThreads) k_umma_dx(const float* __restrict__ dY, int rows, int O,
                                                      const float* __restrict__ Wt, int K, float* __restrict__ dX) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    unsigned char* sa = smem;
    unsigned char* sb = smem + (size_t)kRows * O * 2;
    const int r0 = blockIdx.x * kRows;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) tmem_alloc(&tmem_base, tmem_cols(K));
    if (threadIdx.x == 0) mbar_init(&bar);
    for (int t = threadIdx.x; t < kRows * O; t += blockDim.x) {
        const int rr = t / O, o = t - rr * O;
        const int r = r0 + rr;
        st_bf16(sa, kmajor_off(rr, o, kRows), r < rows ? dY[(size_t)r * O + o] : 0.f);
    }
    for (int t = threadIdx.x; t < K * O; t += blockDim.x) {
        const int o = t / K, k = t - o * K;  // read W row-major, write B[k][o]
        st_bf16(sb, kmajor_off(k, o, K), Wt[(size_t)o * K + k]);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    const bool ok = run_mma(sa, sb, O, K, tmem, &bar);
    if (ok) {
        const int row = warp * 32 + (threadIdx.x & 31);
        const int r = r0 + row;
        for (int c0 = 0; c0 < K; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (r < rows) {
#pragma unroll
                for (int c = 0; c < 16; ++c) dX[(size_t)r * K + c0 + c] = v[c];
            }
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(K));
}

// Weight gradient dW^T[K x O] = X^T dY over one chunk of kDwRows rows per
// CTA: M = the K features in tiles of 128 (zero-padded), N = O, the MMA's
// K dimension = rows, staged kDwSub rows at a time (smem reused after each
// commit completes).  Each CTA writes its partial (Kpad x O, FP32); a second
// kernel sums the partials in CTA order into dW and db.
constexpr int kDwRows = 512;
constexpr int kDwSub = 64;

__global__ void __launch_bounds__(kThreads) k_umma_dw(Parts in, int width, int parts, int rows,
                                                      const float* __restrict__ dY, int O, float* __restrict__ part) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int K = width * parts;
    const int mt = (K + kRows - 1) / kRows;  // 128-feature M tiles
    const int Kp = mt * kRows;
    unsigned char* sa = smem;                            // X^T: Kp features x kDwSub rows
    unsigned char* sb = smem + (size_t)Kp * kDwSub * 2;  // dY^T: O x kDwSub rows
    const int r0 = blockIdx.x * kDwRows;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) tmem_alloc(&tmem_base, tmem_cols(mt * O));
    if (threadIdx.x == 0) mbar_init(&bar);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    bool ok = true;
    int phase = 0;
    for (int c0 = 0; c0 < kDwRows && r0 + c0 < rows; c0 += kDwSub) {
        for (int t = threadIdx.x; t < Kp * kDwSub; t += blockDim.x) {
            const int rr = t / Kp, f = t - rr * Kp;  // consecutive threads: consecutive features of one row
            const int r = r0 + c0 + rr;
            float v = 0.f;
            if (f < K && r < rows) {
                const int p = f / width, col = f - p * width;
                const int src = in.idx[p] ? in.idx[p][r] : r;
                v = in.p[p][(size_t)src * width + col];
            }
            st_bf16(sa, kmajor_off(f, rr, Kp), v);
        }
        for (int t = threadIdx.x; t < O * kDwSub; t += blockDim.x) {
            const int rr = t / O, o = t - rr * O;
            const int r = r0 + c0 + rr;
            st_bf16(sb, kmajor_off(o, rr, O), r < rows ? dY[(size_t)r * O + o] : 0.f);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        fence_after();
        if (threadIdx.x == 0) {
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
            const uint32_t lbo_a = (uint32_t)(Kp / 8) * 128, lbo_b = (uint32_t)(O / 8) * 128;
            const uint32_t idesc = make_idesc(kRows, O);
            for (int m = 0; m < mt; ++m)
                for (int ks = 0; ks < kDwSub / 16; ++ks) {
                    // A rows [m*128, m*128+128): 16 core-matrix groups further along M (SBO = 128 B each)
                    const uint64_t da = make_desc(a0 + (uint32_t)ks * 2 * lbo_a + (uint32_t)m * 16 * 128, lbo_a, 128);
                    const uint64_t db = make_desc(b0 + (uint32_t)ks * 2 * lbo_b, lbo_b, 128);
                    mma_bf16(tmem + (uint32_t)(m * O), da, db, idesc, (c0 > 0 || ks > 0));
                }
            mma_commit(&bar);
        }
        bool w = mbar_wait(&bar, (uint32_t)phase);
        if (!w) {
            atomicExch(&g_umma_error, 1);
            mbar_wait(&bar, (uint32_t)phase);
        }
        ok = (__syncthreads_and(w) != 0) && ok;
        fence_after();
        phase ^= 1;
        if (!ok) break;
    }
    if (ok) {
        const int row = warp * 32 + (threadIdx.x & 31);  // feature within an M tile
        float* out = part + (size_t)blockIdx.x * Kp * O;
        for (int m = 0; m < mt; ++m)
            for (int c0 = 0; c0 < O; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * O + c0), v);
#pragma unroll
                for (int c = 0; c < 16; ++c) out[(size_t)(m * kRows + row) * O + c0 + c] = v[c];
            }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(mt * O));
}

// dW[o][k] += sum_b part[b][k][o];  db[o] += sum_r dY[r][o] (column sums in row order).
__global__ void k_dw_reduce(const float* __restrict__ part, int nparts, int Kp, int K, int O, float* dW) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= K * O) return;
    const int k = t / O, o = t - k * O;
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += part[((size_t)b * Kp + k) * O + o];
    dW[(size_t)o * K + k] += (float)s;
}

// Bias gradient in two fixed-order stages: column sums per kDwRows chunk, then over chunks.
__global__ void k_db_part(const float* __restrict__ dY, int rows, int O, float* __restrict__ dpart) {
    const int o = threadIdx.x;
    if (o >= O) return;
    const int r0 = blockIdx.x * kDwRows, r1 = min(rows, r0 + kDwRows);
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += dY[(size_t)r * O + o];
    dpart[(size_t)blockIdx.x * O + o] = s;
}

__global__ void k_db_reduce(const float* __restrict__ dpart, int nparts, int O, float* db) {
    const int o = threadIdx.x;
    if (o >= O) return;
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += dpart[(size_t)b * O + o];
    db[o] += (float)s;
}

// Shapes the kernels take: M = 128 needs N a multiple of 16 in [16, 256];
// the K (or K-dim O) extent is a whole number of 16-wide MMA slices.
bool umma_gemm_supported(int K, int O) { return K % 16 == 0 && K <= 192 && O % 16 == 0 && O >= 16 && O <= 64; }
bool umma_gemm_dx_supported(int O, int K) { return O % 16 == 0 && O <= 64 && K % 16 == 0 && K >= 16 && K <= 256; }
bool umma_gemm_dw_supported(int K, int O) { return K % 16 == 0 && K <= 256 && O % 16 == 0 && O >= 16 && O <= 64; }
static size_t dw_smem(int K, int O) { return ((size_t)((K + kRows - 1) / kRows) * kRows + O) * kDwSub * 2; }
size_t umma_dw_part_floats(int rows, int K, int O) {
    const size_t nparts = (size_t)((rows + kDwRows - 1) / kDwRows);
    return nparts * ((K + kRows - 1) / kRows) * kRows * O + nparts * O;
}

static size_t fwd_smem(int K, int O) { return (size_t)(kRows + O) * K * 2; }
static size_t dx_smem(int O, int K) { return (size_t)(kRows + K) * O * 2; }

void umma_gemm(const float* const* p, const int* const* idx, int width, int parts, int rows, const float* Wt, int O,
               const float* bias, int relu, const float* resid, float* Y, cudaStream_t st) {
    if (!smem_limit_ok((const void*)k_umma_fwd, fwd_smem(192, 64), "k_umma_fwd shared memory")) return;
    Parts in{};
    for (int i = 0; i < parts; ++i) {
        in.p[i] = p[i];
        in.idx[i] = idx[i];
    }
    const int K = width * parts;
    k_umma_fwd<<<(rows + kRows - 1) / kRows, kThreads, fwd_smem(K, O), st>>>(in, width, parts, rows, Wt, O, bias, relu,
                                                                            resid, Y);
}

void umma_gemm_dx(const float* dY, int rows, int O, const float* Wt, int K, float* dX, cudaStream_t st) {
    if (!smem_limit_ok((const void*)k_umma_dx, dx_smem(64, 256), "k_umma_dx shared memory")) return;
    k_umma_dx<<<(rows + kRows - 1) / kRows, kThreads, dx_smem(O, K), st>>>(dY, rows, O, Wt, K, dX);
}

void umma_gemm_dw(const float* const* p, const int* const* idx, int width, int parts, int rows, const float* dY,
                  int O, float* dW, float* db, float* part, cudaStream_t st) {
    if (!smem_limit_ok((const void*)k_umma_dw, dw_smem(256, 64), "k_umma_dw shared memory")) return;
    Parts in{};
    for (int i = 0; i < parts; ++i) {
        in.p[i] = p[i];
        in.idx[i] = idx[i];
    }
    const int K = width * parts;
    const int nparts = (rows + kDwRows - 1) / kDwRows;
    const int Kp = ((K + kRows - 1) / kRows) * kRows;
    k_umma_dw<<<nparts, kThreads, dw_smem(K, O), st>>>(in, width, parts, rows, dY, O, part);
    k_dw_reduce<<<(K * O + 255) / 256, 256, 0, st>>>(part, nparts, Kp, K, O, dW);
    float* dpart = part + (size_t)nparts * Kp * O;
    k_db_part<<<nparts, 64, 0, st>>>(dY, rows, O, dpart);
    k_db_reduce<<<1, 64, 0, st>>>(dpart, nparts, O, db);
}

int umma_error() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_umma_error, sizeof(int)) != cudaSuccess) return -1;
    if (v) {
        const int z = 0;
        cudaMemcpyToSymbol(g_umma_error, &z, sizeof(int));
    }
    return v;
}

}  // namespace fsd
