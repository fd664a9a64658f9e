// Near-field block preconditioner G ~ (R_FU^pruned + relaxer D)^-1
// (Precondition.cu / Helper_Precondition.cu of the reference).
//
//  1. pruned graph: each particle with itself and its neighbours closer than
//     rp = 2.1, sorted by index (Precondition_GetPrunedNlist_kernel);
//  2. R_FU restricted to that graph as 6x6 blocks (Precondition_RFU_kernel),
//     with relaxer * {1,1,1,4/3,4/3,4/3} added to the diagonal
//     (Precondition_AddIdentity_kernel);
//  3. reverse Cuthill-McKee ordering of the particle graph on the host
//     (genrcm, rcm.cpp:1009, restated in rcm_order below);
//  4. incomplete Cholesky with zero fill.  The scalar IC(0) of the reference
//     on a pattern made of dense 6x6 blocks equals block IC(0), which is what
//     is computed here, with FP64 arithmetic and pivots; a non-positive pivot
//     doubles the relaxer and refactors (Precondition.cu:1457-1489);
//  5. forward / backward block triangular solves, scheduled by dependency
//     level (one launch per level).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_solver.h"

namespace fsd {

struct IChol {
    int N = 0;
    // device
    unsigned* pn = nullptr;      // pruned count per particle (self included)
    unsigned* plist = nullptr;   // N x kPrunedCap, sorted
    int* p_over = nullptr;       // overflow flag
    float* blocks = nullptr;     // assembled blocks, original row order: N x kPrunedCap x 36
    int* perm = nullptr;         // perm[new] = old
    int* rowptr = nullptr;       // permuted block CSR (N+1)
    int* col = nullptr;          // permuted column (new index), sorted
    int* src = nullptr;          // block slot in `blocks` for each CSR entry
    int* diag = nullptr;         // CSR position of the diagonal per row
    int* tpos = nullptr;         // CSR position of the transposed entry
    float* L = nullptr;          // factor blocks (fp32), per CSR entry, row-major 6x6
    float* Linv = nullptr;       // inverse of the diagonal factor block per row
    int* fail = nullptr;         // factorisation failure flag
    int* lev_rows = nullptr;     // rows sorted by forward level
    int* blev_rows = nullptr;    // rows sorted by backward level
    float* ty = nullptr;         // permuted work vector (6N)
    float* tz = nullptr;
    int nnzb_cap = 0;
    // host
    std::vector<int> lev_ptr, blev_ptr;
    std::vector<unsigned> h_pn, h_plist;
    int nnzb = 0;
    int* h_fail = nullptr;
};

// ------------------------------------------------------------ pruned graph
__global__ void k_prune(const float4* __restrict__ pos, int N, Box b, const unsigned* __restrict__ nneigh,
                        const unsigned* __restrict__ nlist, int stride, float rp2, unsigned* pn, unsigned* plist,
                        int* over) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 pi = pos[i];
    unsigned* row = plist + (size_t)i * kPrunedCap;
    unsigned cnt = 1;
    row[0] = i;
    const unsigned nn = nneigh[i];
    for (unsigned q = 0; q < nn; ++q) {
        const unsigned j = nlist[(size_t)i * stride + q];
        const float4 pj = pos[j];
        const float3 r = min_image(make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z), b);
        if (r.x * r.x + r.y * r.y + r.z * r.z < rp2) {
            if (cnt < kPrunedCap) row[cnt] = j;
            ++cnt;
        }
    }
    if (cnt > kPrunedCap) {
        atomicMax(over, (int)cnt);
        cnt = kPrunedCap;
    }
    for (unsigned a = 1; a < cnt; ++a) {
        const unsigned key = row[a];
        int c = (int)a - 1;
        while (c >= 0 && row[c] > key) {
            row[c + 1] = row[c];
            --c;
        }
        row[c + 1] = key;
    }
    pn[i] = cnt;
}

// Assemble the 6x6 blocks of particle i's pruned row (Precondition.cu:530-836):
//   neighbour block  [[A12, B12], [B12, C12]],  B12 = YB12 eps(r)
//   self block       sum over pruned neighbours [[A11, -B11], [B11, C11]]
// with the table's first row for r <= 2 + 1e-4, then relaxer on the diagonal.
__global__ void k_assemble(const float4* __restrict__ pos, int N, Box b, const unsigned* __restrict__ pn,
                           const unsigned* __restrict__ plist, ResTable tab, float rp, float relaxer, float* blocks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 pi = pos[i];
    const unsigned cnt = pn[i];
    const unsigned* row = plist + (size_t)i * kPrunedCap;
    float self[36];
#pragma unroll
    for (int k = 0; k < 36; ++k) self[k] = 0.0f;
    int self_slot = 0;
    const float rp2 = rp * rp;
    for (unsigned s = 0; s < cnt; ++s) {
        const unsigned j = row[s];
        float* blk = blocks + ((size_t)i * kPrunedCap + s) * 36;
        if (j == (unsigned)i) {
            self_slot = s;
            continue;
        }
        const float4 pj = pos[j];
        const float3 R = min_image(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), b);
        const float d2 = R.x * R.x + R.y * R.y + R.z * R.z;
        float c[10];
        if (!(d2 < rp2)) {
#pragma unroll
            for (int k = 0; k < 36; ++k) blk[k] = 0.0f;
            continue;
        }
        const float dist = sqrtf(d2);
        if ((double)dist <= (2.0 + (double)kResMin)) {
#pragma unroll
            for (int k = 0; k < 10; ++k) c[k] = __ldg(tab.vals + k);
        } else {
            const float sv = (float)(((double)dist - 2.0) / (double)kResMin);
            const int ind = (int)(log10f(sv) / kResDr);
            const float dl = __ldg(tab.dist + ind), du = __ldg(tab.dist + ind + 1);
            const float fac = (dist - dl) / (du - dl);
#pragma unroll
            for (int k = 0; k < 10; ++k) {
                const float lo = __ldg(tab.vals + 22 * ind + k), hi = __ldg(tab.vals + 22 * (ind + 1) + k);
                c[k] = lo + (hi - lo) * fac;
            }
        }
        const float XA11 = c[0], XA12 = c[1], YA11 = c[2], YA12 = c[3], YB11 = c[4], YB12 = c[5];
        const float XC11 = c[6], XC12 = c[7], YC11 = c[8], YC12 = c[9];
        const float r[3] = {R.x / dist, R.y / dist, R.z / dist};
        const float epsr[3][3] = {{0.0f, r[2], -r[1]}, {-r[2], 0.0f, r[0]}, {r[1], -r[0], 0.0f}};
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
                const float rr = r[ii] * r[jj];
                const float Imrr = (ii == jj ? 1.0f : 0.0f) - rr;
                const float An = XA12 * rr + YA12 * Imrr, As = XA11 * rr + YA11 * Imrr;
                const float Bn = YB12 * epsr[ii][jj], Bs = YB11 * epsr[ii][jj];
                const float Cn = XC12 * rr + YC12 * Imrr, Cs = XC11 * rr + YC11 * Imrr;
                blk[ii * 6 + jj] = An;
                blk[ii * 6 + jj + 3] = Bn;
                blk[(ii + 3) * 6 + jj] = Bn;
                blk[(ii + 3) * 6 + jj + 3] = Cn;
                self[ii * 6 + jj] += As;
                self[ii * 6 + jj + 3] += -Bs;
                self[(ii + 3) * 6 + jj] += Bs;
                self[(ii + 3) * 6 + jj + 3] += Cs;
            }
        }
    }
    float* sb = blocks + ((size_t)i * kPrunedCap + self_slot) * 36;
#pragma unroll
    for (int k = 0; k < 36; ++k) sb[k] = self[k];
#pragma unroll
    for (int d = 0; d < 6; ++d) sb[d * 7] += relaxer * ((d < 3) ? 1.0f : 1.33333333f);
}

// ------------------------------------------------------------- factorisation
// Block row p of the permuted matrix, rows of one level at a time.
//   L_pq = (B_pq - sum_{k<q} L_pk L_qk^T) L_qq^-T   for q < p in the pattern
//   L_pp = chol(B_pp - sum_{k<p} L_pk L_pk^T)
// FP64 throughout; a non-positive or non-finite pivot sets *fail.
__device__ void chol6(double* A, bool* ok) {
    for (int j = 0; j < 6; ++j) {
        double d = A[j * 6 + j];
        for (int k = 0; k < j; ++k) d -= A[j * 6 + k] * A[j * 6 + k];
        if (!(d > 0.0)) {
            *ok = false;
            d = 1.0;
        }
        d = sqrt(d);
        A[j * 6 + j] = d;
        for (int i = j + 1; i < 6; ++i) {
            double v = A[i * 6 + j];
            for (int k = 0; k < j; ++k) v -= A[i * 6 + k] * A[j * 6 + k];
            A[i * 6 + j] = v / d;
        }
        for (int k = j + 1; k < 6; ++k) A[j * 6 + k] = 0.0;
    }
}

__global__ void k_factor_level(const int* __restrict__ rows, int nrows, const int* __restrict__ rowptr,
                               const int* __restrict__ col, const int* __restrict__ src, const int* __restrict__ diag,
                               const float* __restrict__ blocks, float* L, float* Linv, int* fail) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    const int p = rows[t];
    const int b = rowptr[p], dp = diag[p];
    double acc[36];
    for (int e = b; e <= dp; ++e) {
        const int q = col[e];
        const float* B = blocks + (size_t)src[e] * 36;
        for (int k = 0; k < 36; ++k) acc[k] = (double)B[k];
        // subtract sum_{k < q} L_pk L_qk^T over the common pattern
        const int bq = rowptr[q], dq = diag[q];
        int ip = b, iq = bq;
        while (ip < e && iq < dq) {
            const int cp = col[ip], cq = col[iq];
            if (cp == cq) {
                const float* Lp = L + (size_t)ip * 36;
                const float* Lq = L + (size_t)iq * 36;
                for (int r = 0; r < 6; ++r)
                    for (int c = 0; c < 6; ++c) {
                        double s = 0.0;
                        for (int k = 0; k < 6; ++k) s += (double)Lp[r * 6 + k] * (double)Lq[c * 6 + k];
                        acc[r * 6 + c] -= s;
                    }
                ++ip;
                ++iq;
            } else if (cp < cq) {
                ++ip;
            } else {
                ++iq;
            }
        }
        float* out = L + (size_t)e * 36;
        if (e < dp) {
            // acc <- acc * L_qq^-T : solve X L_qq^T = acc row by row
            const float* Lqq = L + (size_t)dq * 36;
            for (int r = 0; r < 6; ++r) {
                for (int c = 0; c < 6; ++c) {
                    double v = acc[r * 6 + c];
                    for (int k = 0; k < c; ++k) v -= acc[r * 6 + k] * (double)Lqq[c * 6 + k];
                    acc[r * 6 + c] = v / (double)Lqq[c * 6 + c];
                }
            }
            for (int k = 0; k < 36; ++k) out[k] = (float)acc[k];
        } else {
            bool ok = true;
            chol6(acc, &ok);
            if (!ok) atomicExch(fail, 1);
            for (int k = 0; k < 36; ++k) out[k] = (float)acc[k];
            // inverse of the lower-triangular factor, forward substitution on I
            double inv[36];
            for (int k = 0; k < 36; ++k) inv[k] = 0.0;
            for (int c = 0; c < 6; ++c) {
                for (int r = c; r < 6; ++r) {
                    double v = (r == c) ? 1.0 : 0.0;
                    for (int k = c; k < r; ++k) v -= acc[r * 6 + k] * inv[k * 6 + c];
                    inv[r * 6 + c] = v / acc[r * 6 + r];
                }
            }
            float* li = Linv + (size_t)p * 36;
            for (int k = 0; k < 36; ++k) li[k] = (float)inv[k];
        }
    }
}

// ---------------------------------------------------------------- solves
// Forward: z_p = Linv_pp (t_p - sum_{q<p} L_pq z_q), on permuted vectors.
__global__ void k_fwd_level(const int* __restrict__ rows, int nrows, const int* __restrict__ rowptr,
                            const int* __restrict__ col, const int* __restrict__ diag, const float* __restrict__ L,
                            const float* __restrict__ Linv, const float* __restrict__ t, float* z) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int p = rows[k];
    float v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = t[6 * p + c];
    for (int e = rowptr[p]; e < diag[p]; ++e) {
        const int q = col[e];
        const float* B = L + (size_t)e * 36;
        float zq[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) zq[c] = z[6 * q + c];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 6; ++c) s += B[r * 6 + c] * zq[c];
            v[r] -= s;
        }
    }
    const float* Li = Linv + (size_t)p * 36;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c <= r; ++c) s += Li[r * 6 + c] * v[c];
        z[6 * p + r] = s;
    }
}

// Backward: x_p = Linv_pp^T (z_p - sum_{q>p} L_qp^T x_q).
__global__ void k_bwd_level(const int* __restrict__ rows, int nrows, const int* __restrict__ rowptr,
                            const int* __restrict__ col, const int* __restrict__ diag, const int* __restrict__ tpos,
                            const float* __restrict__ L, const float* __restrict__ Linv, const float* __restrict__ z,
                            float* x) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int p = rows[k];
    float v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = z[6 * p + c];
    for (int e = diag[p] + 1; e < rowptr[p + 1]; ++e) {
        const int q = col[e];
        const float* B = L + (size_t)tpos[e] * 36;  // L_qp
        float xq[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) xq[c] = x[6 * q + c];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 6; ++c) s += B[c * 6 + r] * xq[c];
            v[r] -= s;
        }
    }
    const float* Li = Linv + (size_t)p * 36;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        float s = 0.0f;
#pragma unroll
        for (int c = r; c < 6; ++c) s += Li[c * 6 + r] * v[c];
        x[6 * p + r] = s;
    }
}

__global__ void k_permute(const float* __restrict__ in, float* __restrict__ out, const int* __restrict__ perm, int N,
                          int dir) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 6 * N) return;
    const int p = k / 6, c = k % 6;
    if (dir > 0)
        out[k] = in[6 * perm[p] + c];  // to permuted order
    else
        out[6 * perm[p] + c] = in[k];  // back to original order
}

// -------------------------------------------------------------- host RCM
namespace {
// Breadth-first level structure from root over unmasked nodes; returns the
// number of levels, nodes in `order`, level starts in `lstart`.
int level_structure(int root, const std::vector<int>& rp, const std::vector<int>& cl, std::vector<char>& mask,
                    std::vector<int>& order, std::vector<int>& lstart) {
    order.clear();
    lstart.clear();
    order.push_back(root);
    mask[root] = 0;
    size_t lb = 0;
    int nl = 0;
    for (;;) {
        const size_t le = order.size();
        lstart.push_back((int)lb);
        ++nl;
        for (size_t i = lb; i < le; ++i) {
            const int v = order[i];
            for (int e = rp[v]; e < rp[v + 1]; ++e) {
                const int u = cl[e];
                if (mask[u]) {
                    mask[u] = 0;
                    order.push_back(u);
                }
            }
        }
        if (order.size() == le) break;
        lb = le;
    }
    lstart.push_back((int)order.size());
    for (int v : order) mask[v] = 1;
    return nl;
}
}  // namespace

void rcm_order(int n, const std::vector<int>& rp, const std::vector<int>& cl, std::vector<int>& perm) {
    std::vector<char> mask(n, 1);
    std::vector<int> order, lstart, deg(n, 0);
    perm.clear();
    perm.reserve(n);
    for (int start = 0; start < n; ++start) {
        if (!mask[start]) continue;
        // Pseudo-peripheral root (George & Liu).
        int root = start;
        int nl = level_structure(root, rp, cl, mask, order, lstart);
        const int csize = (int)order.size();
        if (nl > 1 && nl != csize) {
            for (;;) {
                int mindeg = csize;
                const int ls = lstart[nl - 1];
                root = order[ls];
                for (int k = ls; k < csize; ++k) {
                    const int v = order[k];
                    int d = 0;
                    for (int e = rp[v]; e < rp[v + 1]; ++e) d += mask[cl[e]] > 0;
                    if (d < mindeg) {
                        root = v;
                        mindeg = d;
                    }
                }
                std::vector<int> o2, l2;
                const int nl2 = level_structure(root, rp, cl, mask, o2, l2);
                if (nl2 <= nl) break;
                nl = nl2;
                order.swap(o2);
                lstart.swap(l2);
                if (csize <= nl) break;
            }
        }
        // Degrees within the component (unmasked neighbours, self loops counted).
        level_structure(root, rp, cl, mask, order, lstart);
        for (int v : order) {
            int d = 0;
            for (int e = rp[v]; e < rp[v + 1]; ++e) d += mask[cl[e]] != 0;
            deg[v] = d;
        }
        // Cuthill-McKee: breadth first, each node's new neighbours by increasing degree.
        const size_t base = perm.size();
        perm.push_back(root);
        mask[root] = 0;
        size_t lvlend = base, lnbr = base + 1;
        while (lvlend < lnbr) {
            const size_t lbegin = lvlend;
            lvlend = lnbr;
            for (size_t i = lbegin; i < lvlend; ++i) {
                const int v = perm[i];
                const size_t fnbr = perm.size();
                for (int e = rp[v]; e < rp[v + 1]; ++e) {
                    const int u = cl[e];
                    if (mask[u]) {
                        mask[u] = 0;
                        perm.push_back(u);
                    }
                }
                // stable insertion sort of perm[fnbr..) by degree
                for (size_t k = fnbr + 1; k < perm.size(); ++k) {
                    const int key = perm[k];
                    size_t l = k;
                    while (l > fnbr && deg[perm[l - 1]] > deg[key]) {
                        perm[l] = perm[l - 1];
                        --l;
                    }
                    perm[l] = key;
                }
                lnbr = perm.size();
            }
        }
        std::reverse(perm.begin() + base, perm.end());
    }
}

// ------------------------------------------------------------ host driver
int precond_alloc(fsd_handle* h) {
    IChol* ic = new IChol();
    h->ichol = ic;
    const int N = h->p.N;
    ic->N = N;
    ic->nnzb_cap = N * kPrunedCap;
    FSD_CHECK_CUDA(cudaMalloc(&ic->pn, sizeof(unsigned) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->plist, sizeof(unsigned) * (size_t)N * kPrunedCap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->p_over, sizeof(int)));
    FSD_CHECK_CUDA(cudaMalloc(&ic->blocks, sizeof(float) * 36 * (size_t)N * kPrunedCap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->perm, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->rowptr, sizeof(int) * (N + 1)));
    FSD_CHECK_CUDA(cudaMalloc(&ic->col, sizeof(int) * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->src, sizeof(int) * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->diag, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->tpos, sizeof(int) * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->L, sizeof(float) * 36 * (size_t)ic->nnzb_cap));
    FSD_CHECK_CUDA(cudaMalloc(&ic->Linv, sizeof(float) * 36 * (size_t)N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->fail, sizeof(int)));
    FSD_CHECK_CUDA(cudaMalloc(&ic->lev_rows, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->blev_rows, sizeof(int) * N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->ty, sizeof(float) * 6 * (size_t)N));
    FSD_CHECK_CUDA(cudaMalloc(&ic->tz, sizeof(float) * 6 * (size_t)N));
    FSD_CHECK_CUDA(cudaMallocHost(&ic->h_fail, sizeof(int) * 2));
    return FSD_OK;
}

void precond_free(fsd_handle* h) {
    IChol* ic = (IChol*)h->ichol;
    if (!ic) return;
    void* ptrs[] = {ic->pn, ic->plist, ic->p_over, ic->blocks, ic->perm, ic->rowptr, ic->col, ic->src, ic->diag,
                    ic->tpos, ic->L, ic->Linv, ic->fail, ic->lev_rows, ic->blev_rows, ic->ty, ic->tz};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (ic->h_fail) cudaFreeHost(ic->h_fail);
    delete ic;
    h->ichol = nullptr;
}

// Build the pattern, ordering and levels from the pruned graph (host), then
// factor with the current relaxer, doubling it on failure.
int precond_build(fsd_handle* h, const float4* pos) {
    IChol* ic = (IChol*)h->ichol;
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    if (h->p.precond == FSD_PRECOND_NONE) {
        h->pc_valid = true;
        return FSD_OK;
    }
    FSD_CHECK_CUDA(cudaMemsetAsync(ic->p_over, 0, sizeof(int), st));
    k_prune<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, h->w.nneigh, h->w.nlist, h->w.nl_stride,
                                             h->p.rp * h->p.rp, ic->pn, ic->plist, ic->p_over);
    ic->h_pn.resize(N);
    ic->h_plist.resize((size_t)N * kPrunedCap);
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_pn.data(), ic->pn, sizeof(unsigned) * N, cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_plist.data(), ic->plist, sizeof(unsigned) * (size_t)N * kPrunedCap,
                                   cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_fail, ic->p_over, sizeof(int), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    if (ic->h_fail[0] > 0) return FSD_ERR_NLIST_OVERFLOW;
    // Particle graph in CSR (self loops included, rows sorted).
    std::vector<int> rp(N + 1, 0), cl;
    cl.reserve((size_t)N * 6);
    for (int i = 0; i < N; ++i) {
        for (unsigned s = 0; s < ic->h_pn[i]; ++s) cl.push_back((int)ic->h_plist[(size_t)i * kPrunedCap + s]);
        rp[i + 1] = (int)cl.size();
    }
    std::vector<int> perm, inv(N);
    rcm_order(N, rp, cl, perm);
    for (int p = 0; p < N; ++p) inv[perm[p]] = p;
    // Permuted block CSR with sorted new-index columns.
    std::vector<int> prow(N + 1, 0), pcol, psrc, pdiag(N), ptpos;
    pcol.reserve(cl.size());
    psrc.reserve(cl.size());
    std::vector<std::pair<int, int>> tmp;
    for (int p = 0; p < N; ++p) {
        const int i = perm[p];
        tmp.clear();
        for (int e = rp[i]; e < rp[i + 1]; ++e) tmp.emplace_back(inv[cl[e]], i * kPrunedCap + (e - rp[i]));
        std::sort(tmp.begin(), tmp.end());
        for (auto& t : tmp) {
            if (t.first == p) pdiag[p] = (int)pcol.size();
            pcol.push_back(t.first);
            psrc.push_back(t.second);
        }
        prow[p + 1] = (int)pcol.size();
    }
    const int nnzb = (int)pcol.size();
    ic->nnzb = nnzb;
    ptpos.assign(nnzb, -1);
    for (int p = 0; p < N; ++p)
        for (int e = prow[p]; e < prow[p + 1]; ++e) {
            const int q = pcol[e];
            // position of (q, p) in row q (pattern is symmetric)
            const int* b = pcol.data() + prow[q];
            const int* en = pcol.data() + prow[q + 1];
            const int* f = std::lower_bound(b, en, p);
            ptpos[e] = (f != en && *f == p) ? (int)(f - pcol.data()) : -1;
        }
    // Dependency levels (forward and backward).
    std::vector<int> lev(N, 0), blev(N, 0);
    int nlev = 0, nblev = 0;
    for (int p = 0; p < N; ++p) {
        int l = 0;
        for (int e = prow[p]; e < pdiag[p]; ++e) l = std::max(l, lev[pcol[e]] + 1);
        lev[p] = l;
        nlev = std::max(nlev, l + 1);
    }
    for (int p = N - 1; p >= 0; --p) {
        int l = 0;
        for (int e = pdiag[p] + 1; e < prow[p + 1]; ++e) l = std::max(l, blev[pcol[e]] + 1);
        blev[p] = l;
        nblev = std::max(nblev, l + 1);
    }
    auto bucket = [N](const std::vector<int>& lv, int nl, std::vector<int>& ptr, std::vector<int>& rows) {
        ptr.assign(nl + 1, 0);
        for (int p = 0; p < N; ++p) ptr[lv[p] + 1]++;
        for (int l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
        rows.resize(N);
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int p = 0; p < N; ++p) rows[fill[lv[p]]++] = p;
    };
    std::vector<int> lrows, brows;
    bucket(lev, nlev, ic->lev_ptr, lrows);
    bucket(blev, nblev, ic->blev_ptr, brows);
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->perm, perm.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->rowptr, prow.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->col, pcol.data(), sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->src, psrc.data(), sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->diag, pdiag.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->tpos, ptpos.data(), sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->lev_rows, lrows.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    FSD_CHECK_CUDA(cudaMemcpyAsync(ic->blev_rows, brows.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    h->info.ichol_attempts = 0;
    // Factor, doubling the relaxer after each failure (Precondition.cu:1457-1489).
    for (int attempt = 0; attempt < 24; ++attempt) {
        k_assemble<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, ic->pn, ic->plist,
                                                   ResTable{h->d_res_dist, h->d_res_vals}, h->p.rp, h->ichol_relaxer,
                                                   ic->blocks);
        FSD_CHECK_CUDA(cudaMemsetAsync(ic->fail, 0, sizeof(int), st));
        for (int l = 0; l < nlev; ++l) {
            const int n = ic->lev_ptr[l + 1] - ic->lev_ptr[l];
            k_factor_level<<<(n + 63) / 64, 64, 0, st>>>(ic->lev_rows + ic->lev_ptr[l], n, ic->rowptr, ic->col,
                                                        ic->src, ic->diag, ic->blocks, ic->L, ic->Linv, ic->fail);
        }
        FSD_CHECK_CUDA(cudaMemcpyAsync(ic->h_fail, ic->fail, sizeof(int), cudaMemcpyDeviceToHost, st));
        FSD_CHECK_CUDA(cudaStreamSynchronize(st));
        h->info.ichol_attempts = attempt + 1;
        if (!ic->h_fail[0]) {
            h->info.ichol_relaxer = h->ichol_relaxer;
            h->pc_valid = true;
            return FSD_OK;
        }
        h->ichol_relaxer *= 2.0f;
    }
    return FSD_ERR_ICHOL;
}

int precond_G(fsd_handle* h, const float* t, float* y) {
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    if (h->p.precond == FSD_PRECOND_NONE) {
        FSD_CHECK_CUDA(cudaMemcpyAsync(y, t, sizeof(float) * 6 * N, cudaMemcpyDeviceToDevice, st));
        return FSD_OK;
    }
    IChol* ic = (IChol*)h->ichol;
    k_permute<<<(6 * N + 255) / 256, 256, 0, st>>>(t, ic->ty, ic->perm, N, 1);
    const int nlev = (int)ic->lev_ptr.size() - 1;
    for (int l = 0; l < nlev; ++l) {
        const int n = ic->lev_ptr[l + 1] - ic->lev_ptr[l];
        k_fwd_level<<<(n + 127) / 128, 128, 0, st>>>(ic->lev_rows + ic->lev_ptr[l], n, ic->rowptr, ic->col, ic->diag,
                                                     ic->L, ic->Linv, ic->ty, ic->tz);
    }
    const int nblev = (int)ic->blev_ptr.size() - 1;
    for (int l = 0; l < nblev; ++l) {
        const int n = ic->blev_ptr[l + 1] - ic->blev_ptr[l];
        k_bwd_level<<<(n + 127) / 128, 128, 0, st>>>(ic->blev_rows + ic->blev_ptr[l], n, ic->rowptr, ic->col,
                                                     ic->diag, ic->tpos, ic->L, ic->Linv, ic->tz, ic->ty);
    }
    k_permute<<<(6 * N + 255) / 256, 256, 0, st>>>(ic->ty, y, ic->perm, N, -1);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

}  // namespace fsd
