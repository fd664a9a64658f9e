// Sparse approximate inverse of A = R_FU^pruned + D on the two-hop pattern of
// the pruned contact graph (the base of FSD_PRECOND_LEARNED).
//
// For each particle c, S_c = {c} + pruned neighbours + their pruned
// neighbours (first kSpaiCap, in that order).  The columns of A restricted to
// S_c give the least-squares problem
//     min || A[:, S_c] X_c - E_c ||_F,     E_c = the 6 columns of particle c,
// whose normal equations (A^2)[S_c, S_c] X_c = A[S_c, c] are assembled and
// solved by Cholesky in FP64, one CTA per particle with the packed normal
// matrix in shared memory.  X_c is column c of a right approximate inverse,
// A G ~ I (Grote and Huckle's SPAI with a fixed pattern), which suits the
// right-preconditioned inner GMRES.
// Launches are bucketed by |S_c| so small systems share an SM.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_profile.h"
#include "fsd_solver.h"

namespace fsd {

namespace {
// Buckets of set sizes (particles per two-hop set), so that each launch sizes
// its shared memory for its largest set; the larger sets get 256 threads.
constexpr int kBuckets = 6;
constexpr int kBucketMax[kBuckets] = {12, 16, 20, 24, 28, kSpaiCap};
__host__ __device__ constexpr int bucket_of(int n) { return n <= 12 ? 0 : (n <= 28 ? (n - 9) / 4 : 5); }
constexpr int bucket_threads(int b) { return kBucketMax[b] > 16 ? 256 : 128; }

inline size_t spai_smem(int m) {  // packed FP64 lower triangle + 6 right-hand sides + inverse pivots + the set
    const size_t n = 6 * (size_t)m;
    return sizeof(double) * (n * (n + 1) / 2 + 7 * n) + sizeof(int) * kSpaiCap;
}
}  // namespace

// Two-hop sets (c first, then the 1-hop list, then new 2-hop members in list
// order), truncated at kSpaiCap; bucket lists for the solve launches.
__global__ void k_spai_sets(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist, int N, int* sets,
                            unsigned* ns, unsigned* bucket_cnt, int* bucket_list, int* truncated) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    int* S = sets + (size_t)c * kSpaiCap;
    int n = 0;
    bool over = false;
    S[n++] = c;
    const unsigned* row = plist + (size_t)c * kPrunedCap;
    for (unsigned q = 0; q < pn[c]; ++q)
        if ((int)row[q] != c) {
            if (n < kSpaiCap) S[n++] = (int)row[q];
            else over = true;
        }
    const int n1 = n;
    for (int a = 1; a < n1; ++a) {
        const int k = S[a];
        const unsigned* rk = plist + (size_t)k * kPrunedCap;
        for (unsigned q = 0; q < pn[k]; ++q) {
            const int s = (int)rk[q];
            bool seen = false;
            for (int b = 0; b < n; ++b)
                if (S[b] == s) {
                    seen = true;
                    break;
                }
            if (seen) continue;
            if (n < kSpaiCap) S[n++] = s;
            else over = true;
        }
    }
    ns[c] = (unsigned)n;
    if (over) atomicAdd(truncated, 1);
    const int b = bucket_of(n);
    const unsigned slot = atomicAdd(bucket_cnt + b, 1u);
    bucket_list[(size_t)b * N + slot] = c;
}

__device__ __forceinline__ size_t tri(int i, int j) { return (size_t)i * (i + 1) / 2 + j; }  // i >= j

// Block (s, k) of A from the pruned list of s (k must be on it), or null.
__device__ __forceinline__ const float* a_block(const unsigned* pn, const unsigned* plist, const float* A, int s,
                                                int k) {
    const unsigned* row = plist + (size_t)s * kPrunedCap;
    const unsigned n = pn[s];
    for (unsigned q = 0; q < n; ++q)
        if ((int)row[q] == k) return A + ((size_t)s * kPrunedCap + q) * 36;
    return nullptr;
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) k_spai_solve(const unsigned* __restrict__ pn,
                                                             const unsigned* __restrict__ plist,
                                                             const float* __restrict__ A,
                                                             const int* __restrict__ sets,
                                                             const unsigned* __restrict__ ns,
                                                             const unsigned* __restrict__ bucket_cnt,
                                                             const int* __restrict__ bucket_list, int bucket, int N,
                                                             const int* __restrict__ rowptr, int* g_col, float* g_val,
                                                             int* fail) {
    if (blockIdx.x >= bucket_cnt[bucket]) return;
    const int c = bucket_list[(size_t)bucket * N + blockIdx.x];
    extern __shared__ double sm[];
    const int m = (int)ns[c];
    const int n = 6 * m;
    double* H = sm;                               // packed lower triangle, n(n+1)/2
    double* R = sm + (size_t)n * (n + 1) / 2;     // n x 6, row-major
    double* dinv = R + 6 * (size_t)n;             // 1 / L_jj
    int* S = (int*)(dinv + n);
    for (int a = threadIdx.x; a < m; a += blockDim.x) S[a] = sets[(size_t)c * kSpaiCap + a];
    __syncthreads();
    // Normal matrix: H[a][b] = sum_k A_{s_a k} A_{s_b k}^T over k in both pruned lists (b <= a).
    const int npairs = m * (m + 1) / 2;
    for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
        int a = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while ((a + 1) * (a + 2) / 2 <= t) ++a;
        while (a * (a + 1) / 2 > t) --a;
        const int b = t - a * (a + 1) / 2;
        const int sa = S[a], sb = S[b];
        const unsigned* ra = plist + (size_t)sa * kPrunedCap;
        const unsigned* rb = plist + (size_t)sb * kPrunedCap;
        const unsigned na = pn[sa], nb = pn[sb];
        // three rows of the 6x6 block per pass (18 FP64 accumulators in registers)
        for (int r0 = 0; r0 < 6; r0 += 3) {
            double acc[3][6];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int q = 0; q < 6; ++q) acc[r][q] = 0.0;
            unsigned ia = 0, ib = 0;
            while (ia < na && ib < nb) {
                const unsigned ka = ra[ia], kb = rb[ib];
                if (ka == kb) {
                    const float* Pa = A + ((size_t)sa * kPrunedCap + ia) * 36 + r0 * 6;
                    const float* Pb = A + ((size_t)sb * kPrunedCap + ib) * 36;
                    float pa[18], pb[36];
#pragma unroll
                    for (int u = 0; u < 18; ++u) pa[u] = Pa[u];
#pragma unroll
                    for (int u = 0; u < 36; ++u) pb[u] = Pb[u];
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int q = 0; q < 6; ++q) {
                            double v = 0.0;
#pragma unroll
                            for (int u = 0; u < 6; ++u) v += (double)pa[r * 6 + u] * (double)pb[q * 6 + u];
                            acc[r][q] += v;
                        }
                    ++ia;
                    ++ib;
                } else if (ka < kb) {
                    ++ia;
                } else {
                    ++ib;
                }
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int i = 6 * a + r0 + r;
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const int j = 6 * b + q;
                    if (i >= j) H[tri(i, j)] = acc[r][q];
                }
            }
        }
    }
    // Right-hand sides: R[6a + r][q] = A_{s_a c}[r][q].
    for (int a = threadIdx.x; a < m; a += blockDim.x) {
        const float* blk = a_block(pn, plist, A, S[a], c);
        for (int k = 0; k < 36; ++k) R[(size_t)(6 * a + k / 6) * 6 + k % 6] = blk ? (double)blk[k] : 0.0;
    }
    __syncthreads();
    // Right-looking block Cholesky on the 6x6 blocks of the particles, in
    // place, with the forward substitution L y = R carried along.  Per block
    // column: one thread factors the diagonal block (keeping 1 / L_jj, so
    // the rest multiplies instead of dividing), the rows below take their
    // panel entries (one row per thread) while six threads solve the block's
    // right-hand sides, then the trailing lower triangle and right-hand sides
    // are updated with the work spread evenly over the threads (one entry,
    // or one right-hand-side row, per item).  Three barriers per block column.
    __shared__ int bad;
    __shared__ double bsum[THREADS];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int jb = 0; jb < m; ++jb) {
        const int j0 = 6 * jb;
        if (threadIdx.x == 0) {
            for (int j = j0; j < j0 + 6; ++j) {
                double d = H[tri(j, j)];
                for (int q = j0; q < j; ++q) d -= H[tri(j, q)] * H[tri(j, q)];
                if (!(d > 0.0)) {
                    bad = 1;
                    d = 1.0;
                }
                const double inv = rsqrt(d);
                H[tri(j, j)] = d * inv;
                dinv[j] = inv;
                for (int i = j + 1; i < j0 + 6; ++i) {
                    double v = H[tri(i, j)];
                    for (int q = j0; q < j; ++q) v -= H[tri(i, q)] * H[tri(j, q)];
                    H[tri(i, j)] = v * inv;
                }
            }
        }
        __syncthreads();
        // panel: L[i][j0:j0+6] = H[i][j0:j0+6] L_jj^-T for the rows below
        for (int i = j0 + 6 + threadIdx.x; i < n; i += blockDim.x) {
            double l[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                double v = H[tri(i, j0 + q)];
                for (int p2 = 0; p2 < q; ++p2) v -= l[p2] * H[tri(j0 + q, j0 + p2)];
                l[q] = v * dinv[j0 + q];
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) H[tri(i, j0 + q)] = l[q];
        }
        // right-hand side rows of this block: y = L_jj^-1 R (one column per thread)
        if (threadIdx.x >= blockDim.x - 6) {
            const int c = threadIdx.x - (blockDim.x - 6);
            for (int q = 0; q < 6; ++q) {
                double v = R[(size_t)(j0 + q) * 6 + c];
                for (int p2 = 0; p2 < q; ++p2) v -= H[tri(j0 + q, j0 + p2)] * R[(size_t)(j0 + p2) * 6 + c];
                R[(size_t)(j0 + q) * 6 + c] = v * dinv[j0 + q];
            }
        }
        __syncthreads();
        // trailing update: items [0, T(T+1)/2) are the entries (i, k), k <= i,
        // of the trailing lower triangle (i = j0 + 6 + i', k = j0 + 6 + k');
        // items [T(T+1)/2, T(T+1)/2 + T) are its right-hand-side rows
        const int T = n - j0 - 6;
        const int ntri = T * (T + 1) / 2;
        for (int t = threadIdx.x; t < ntri + T; t += blockDim.x) {
            if (t < ntri) {
                int ip = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
                while ((ip + 1) * (ip + 2) / 2 <= t) ++ip;
                while (ip * (ip + 1) / 2 > t) --ip;
                const int kp = t - ip * (ip + 1) / 2;
                const double* li = H + tri(j0 + 6 + ip, j0);
                const double* lk = H + tri(j0 + 6 + kp, j0);
                H[tri(j0 + 6 + ip, j0 + 6 + kp)] -= li[0] * lk[0] + li[1] * lk[1] + li[2] * lk[2] + li[3] * lk[3] +
                                                    li[4] * lk[4] + li[5] * lk[5];
            } else {
                const int i = j0 + 6 + (t - ntri);
                const double* li = H + tri(i, j0);
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    double v = 0.0;
#pragma unroll
                    for (int q = 0; q < 6; ++q) v += li[q] * R[(size_t)(j0 + q) * 6 + c];
                    R[(size_t)i * 6 + c] -= v;
                }
            }
        }
        __syncthreads();
    }
    // Backward substitution L^T x = y by blocks: the coupling of block jb to
    // the solved blocks below is summed by all threads ((q, c) pairs times
    // kParts row ranges), then the 6x6 triangular solve (one column per thread).
    constexpr int kParts = THREADS / 36;  // 3 with 128 threads, 7 with 256
    for (int jb = m - 1; jb >= 0; --jb) {
        const int j0 = 6 * jb;
        const int t = threadIdx.x;
        const int pc = t % 36, part = t / 36;
        double v = 0.0;
        if (part < kParts) {
            const int q = pc / 6, c = pc % 6;
            for (int i = j0 + 6 + part; i < n; i += kParts) v += H[tri(i, j0 + q)] * R[(size_t)i * 6 + c];
        }
        bsum[t] = v;
        __syncthreads();
        if (t < 36) {
            const int q = t / 6, c = t % 6;
            double sum = 0.0;
#pragma unroll
            for (int k = 0; k < kParts; ++k) sum += bsum[t + 36 * k];
            R[(size_t)(j0 + q) * 6 + c] -= sum;
        }
        __syncthreads();
        if (t < 6) {
            const int c = t;
            for (int q = 5; q >= 0; --q) {
                double w = R[(size_t)(j0 + q) * 6 + c];
                for (int p2 = q + 1; p2 < 6; ++p2) w -= H[tri(j0 + p2, j0 + q)] * R[(size_t)(j0 + p2) * 6 + c];
                R[(size_t)(j0 + q) * 6 + c] = w * dinv[j0 + q];
            }
        }
        __syncthreads();
    }
    // Column c of G: block (s_a, c) = X block a, stored in row s_a at the
    // position of c in that row's set (the sets are mutual unless one was
    // truncated; a block without a slot is dropped).  A failed factorisation
    // (never expected: the normal matrix of a full-rank A[:, S] is SPD) leaves
    // the block-Jacobi inverse in column c.
    if (!bad) {
        for (int a = threadIdx.x; a < m; a += blockDim.x) {
            const int sa = S[a];
            const int* Ss = sets + (size_t)sa * kSpaiCap;
            const int ms = (int)ns[sa];
            int p = -1;
            for (int q = 0; q < ms; ++q)
                if (Ss[q] == c) {
                    p = q;
                    break;
                }
            if (p < 0) continue;
            float* out = g_val + (size_t)(rowptr[sa] + p) * 36;
            for (int k = 0; k < 36; ++k) out[k] = (float)R[(size_t)(6 * a + k / 6) * 6 + k % 6];
        }
    } else if (threadIdx.x == 0) {
        atomicAdd(fail, 1);
        const float* d = a_block(pn, plist, A, c, c);
        double M[6][12];
        for (int r = 0; r < 6; ++r)
            for (int q = 0; q < 12; ++q) M[r][q] = q < 6 ? (double)d[r * 6 + q] : (q - 6 == r ? 1.0 : 0.0);
        for (int k = 0; k < 6; ++k) {
            const double pv = M[k][k] != 0.0 ? 1.0 / M[k][k] : 0.0;
            for (int q = 0; q < 12; ++q) M[k][q] *= pv;
            for (int r = 0; r < 6; ++r)
                if (r != k) {
                    const double f = M[r][k];
                    for (int q = 0; q < 12; ++q) M[r][q] -= f * M[k][q];
                }
        }
        for (int r = 0; r < 6; ++r)
            for (int q = 0; q < 6; ++q) g_val[(size_t)rowptr[c] * 36 + r * 6 + q] = (float)M[r][6 + q];
    }
}

// Column indices of G's rows: row s holds its own set.
__global__ void k_spai_cols(const int* __restrict__ sets, const unsigned* __restrict__ ns,
                            const int* __restrict__ rowptr, int N, int* g_col) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    for (unsigned q = 0; q < ns[s]; ++q) g_col[rowptr[s] + q] = sets[(size_t)s * kSpaiCap + q];
}

int spai_build(fsd_handle* h) {
    LearnedState* s = learned(h);
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    if (!s->sp_sets) {
        FSD_CHECK_CUDA(cudaMalloc(&s->sp_sets, sizeof(int) * (size_t)N * kSpaiCap));
        FSD_CHECK_CUDA(cudaMalloc(&s->sp_size, sizeof(unsigned) * N));
        FSD_CHECK_CUDA(cudaMalloc(&s->sp_rowptr, sizeof(unsigned) * (N + 1)));
        FSD_CHECK_CUDA(cudaMalloc(&s->sp_scan, sizeof(unsigned) * scan_scratch_elems(N)));
        FSD_CHECK_CUDA(cudaMalloc(&s->sp_bucket, sizeof(int) * (size_t)kBuckets * N));
        FSD_CHECK_CUDA(cudaMalloc(&s->sp_cnt, sizeof(unsigned) * (kBuckets + 2)));
        FSD_CHECK_CUDA(cudaMallocHost(&s->sp_host, sizeof(unsigned) * (kBuckets + 2)));
        FSD_CHECK_CUDA(ensure_smem_limit((const void*)k_spai_solve<128>, spai_smem(16)));
        FSD_CHECK_CUDA(ensure_smem_limit((const void*)k_spai_solve<256>, spai_smem(kSpaiCap)));
    }
    // counters: buckets [0, kBuckets), then truncated sets, then failed rows
    FSD_CHECK_CUDA(cudaMemsetAsync(s->sp_cnt, 0, sizeof(unsigned) * (kBuckets + 2), st));
    int* truncated = (int*)(s->sp_cnt + kBuckets);
    int* fail = (int*)(s->sp_cnt + kBuckets + 1);
    count_launch();
    k_spai_sets<<<(N + 127) / 128, 128, 0, st>>>(s->a_pn, s->a_plist, N, s->sp_sets, s->sp_size, s->sp_cnt,
                                                 s->sp_bucket, truncated);
    exclusive_scan(s->sp_size, s->sp_rowptr, N, s->sp_scan, st);
    // block count, truncated sets and the bucket sizes (the launches below are sized by them)
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->sp_host, s->sp_rowptr + N, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->sp_host + 1, s->sp_cnt, sizeof(unsigned) * (kBuckets + 1),
                                   cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    const int nnzb = (int)s->sp_host[0];
    s->sp_truncated = (int)s->sp_host[1 + kBuckets];
    int e = learned_reserve(h, nnzb);
    if (e != FSD_OK) return e;
    FSD_CHECK_CUDA(cudaMemcpyAsync(s->g_rowptr, s->sp_rowptr, sizeof(int) * (N + 1), cudaMemcpyDeviceToDevice, st));
    FSD_CHECK_CUDA(cudaMemsetAsync(s->g_val, 0, sizeof(float) * 36 * (size_t)nnzb, st));
    count_launch();
    k_spai_cols<<<(N + 127) / 128, 128, 0, st>>>(s->sp_sets, s->sp_size, s->g_rowptr, N, s->g_col);
    for (int b = 0; b < kBuckets; ++b) {
        const unsigned cnt = s->sp_host[1 + b];
        if (cnt == 0) continue;
        count_launch();
        if (bucket_threads(b) == 128)
            k_spai_solve<128><<<cnt, 128, spai_smem(kBucketMax[b]), st>>>(
                s->a_pn, s->a_plist, s->a_blocks, s->sp_sets, s->sp_size, s->sp_cnt, s->sp_bucket, b, N,
                s->g_rowptr, s->g_col, s->g_val, fail);
        else
            k_spai_solve<256><<<cnt, 256, spai_smem(kBucketMax[b]), st>>>(
                s->a_pn, s->a_plist, s->a_blocks, s->sp_sets, s->sp_size, s->sp_cnt, s->sp_bucket, b, N,
                s->g_rowptr, s->g_col, s->g_val, fail);
    }
    FSD_CHECK_CUDA(cudaGetLastError());
    s->g_nnzb = nnzb;
    return FSD_OK;
}

}  // namespace fsd
