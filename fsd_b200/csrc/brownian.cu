// Brownian pieces of the velocity path:
//   far field  U_B^ff = sqrt(2kT/dt) (M_wave^1/2 xi + M_real^1/2 psi)
//              (Brownian_FarField.cu:829-1061): a random field on the wave
//              space grid scaled by the square root of the Green's function,
//              plus a Lanczos square root of the real-space mobility;
//   near field F_B^nf = sqrt(2kT/dt) R_FU^1/2 psi (Brownian_NearField.cu:174-464);
//   drift      random finite difference (Integrator.cu:549-718).
//
// Normals come from a counter-based Philox4x32-10 generator (Salmon, Moraes,
// Dror & Shaw, SC'11) keyed by (seed, timestep, stream), so every draw is
// reproducible and independent of launch shape.  Lanczos (Chow & Saad 2014)
// keeps FP32 basis vectors, FP64 alpha/beta, and an FP64 implicit-QL
// eigendecomposition of the tridiagonal matrix on the host.
#include <cmath>
#include <functional>
#include <vector>

#include "fsd_brownian.h"
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_profile.h"
#include "fsd_solver.h"

namespace fsd {

// ----------------------------------------------------------------- Philox
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Four standard normals for counter `idx` of stream (key, step) by Box-Muller.
__device__ __forceinline__ float4 normal4(uint32_t key, uint32_t step, uint32_t stream, uint32_t idx) {
    const uint4 r = philox4x32_10(make_uint4(idx, step, stream, 0x46534442u), make_uint2(key, 0x9E3779B9u ^ stream));
    const float s = 2.3283064365386963e-10f;  // 2^-32
    const float u0 = ((float)r.x + 0.5f) * s, u1 = ((float)r.y + 0.5f) * s;
    const float u2 = ((float)r.z + 0.5f) * s, u3 = ((float)r.w + 0.5f) * s;
    const float a = sqrtf(-2.0f * logf(u0)), b = sqrtf(-2.0f * logf(u2));
    float s1, c1, s2, c2;
    sincospif(2.0f * u1, &s1, &c1);
    sincospif(2.0f * u3, &s2, &c2);
    return make_float4(a * c1, a * s1, b * c2, b * s2);
}

__global__ void k_normals(float* out, size_t n, uint32_t key, uint32_t step, uint32_t stream, float scale) {
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (4 * q >= n) return;
    const float4 z = normal4(key, step, stream, (uint32_t)q);
    const float v[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (4 * q + c < n) out[4 * q + c] = scale * v[c];
}

void gaussian(fsd_handle* h, float* out, size_t n, uint32_t step, uint32_t stream, float scale) {
    const size_t nq = (n + 3) / 4;
    count_launch();
    k_normals<<<(unsigned)((nq + 255) / 256), 256, 0, h->stream>>>(out, n, h->seed_hashed, step, stream, scale);
}

// ----------------------------------------------------- wave-space noise field
// Brownian_FarField_RNG_Grid1of2 / 2of2 (Brownian_FarField.cu:113-374): a
// conjugate-symmetric complex Gaussian field f(k) of variance fac^2 per real
// and imaginary part (fac = sqrt(T / dt / quadW); self-conjugate modes are
// real with variance 2 fac^2), mapped to
//   U(k) = j0(k) sqrt(w(k)) (I - kk) f,   D_ab(k) = i 3 j1(k)/k U_a(k) k_b / j0(k)
// and packed like the Green step's output.  Each mirror pair {k, m(k)} is
// drawn once, so every mode gets independent normals.
__device__ __forceinline__ void noise_map(const float4 tk, const float2* f, float2* o, float sgn) {
    const float ksq = tk.x * tk.x + tk.y * tk.y + tk.z * tk.z;
    const float k = sqrtf(ksq);
    const float B = sqrtf(tk.w);
    const float sk = sinf(k), ck = cosf(k);
    const float SU = sk / k;
    const float SD = sgn * (float)(3.0 * (double)(sk - k * ck) / (double)(ksq * k));
    const float2 kdF = make_float2((tk.x * f[0].x + tk.y * f[1].x + tk.z * f[2].x) / ksq,
                                   (tk.x * f[0].y + tk.y * f[1].y + tk.z * f[2].y) / ksq);
    const float kv[3] = {tk.x, tk.y, tk.z};
    float2 W[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) W[a] = make_float2((f[a].x - kv[a] * kdF.x) * B, (f[a].y - kv[a] * kdF.y) * B);
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = make_float2(SU * W[a].x, SU * W[a].y);
    const int ia[8] = {0, 0, 0, 1, 1, 1, 2, 2};
    const int ib[8] = {0, 1, 2, 0, 1, 2, 0, 1};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float2 Wk = make_float2(W[ia[c]].x * kv[ib[c]], W[ia[c]].y * kv[ib[c]]);
        o[3 + c] = make_float2(-SD * Wk.y, SD * Wk.x);
    }
}

__constant__ int kNzA[6] = {0, 3, 5, 7, 9, 2};
__constant__ int kNzB[6] = {1, 4, 6, 8, 10, -1};

__global__ void k_noise_spectrum(float2* __restrict__ grid, const float4* __restrict__ gridk, int Nx, int Ny, int Nz,
                                 float fac, uint32_t key, uint32_t step, uint32_t stream) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int G = Nx * Ny * Nz;
    if (idx >= G) return;
    const int i = idx / (Ny * Nz), j = (idx / Nz) % Ny, l = idx % Nz;
    const int m = (((Nx - i) % Nx) * Ny + (Ny - j) % Ny) * Nz + (Nz - l) % Nz;
    if (m < idx) return;
    if (idx == 0) {
#pragma unroll
        for (int p = 0; p < 6; ++p) grid[(size_t)p * G] = make_float2(0.f, 0.f);
        return;
    }
    const float4 z0 = normal4(key, step, stream, 2 * (uint32_t)idx);
    const float4 z1 = normal4(key, step, stream, 2 * (uint32_t)idx + 1);
    float2 f[3];
    if (m == idx) {
        const float s2 = 1.414213562373095f * fac;
        f[0] = make_float2(s2 * z0.x, 0.f);
        f[1] = make_float2(s2 * z0.y, 0.f);
        f[2] = make_float2(s2 * z0.z, 0.f);
    } else {
        f[0] = make_float2(fac * z0.x, fac * z0.w);
        f[1] = make_float2(fac * z0.y, fac * z1.x);
        f[2] = make_float2(fac * z0.z, fac * z1.y);
    }
    float2 o[11];
    noise_map(gridk[idx], f, o, 1.0f);
    const bool nyq = (2 * i == Nx) || (2 * j == Ny) || (2 * l == Nz);
    if (nyq) {
        float2 o2[11];
        noise_map(gridk[m], f, o2, -1.0f);
#pragma unroll
        for (int c = 0; c < 11; ++c) o[c] = make_float2(0.5f * (o[c].x + o2[c].x), 0.5f * (o[c].y + o2[c].y));
    }
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        const float2 A = o[kNzA[p]];
        const float2 Bv = (kNzB[p] >= 0) ? o[kNzB[p]] : make_float2(0.f, 0.f);
        grid[(size_t)p * G + idx] = make_float2(A.x - Bv.y, A.y + Bv.x);
        if (m != idx) grid[(size_t)p * G + m] = make_float2(A.x + Bv.y, -A.y + Bv.x);
    }
}

// ------------------------------------------------------------------ vectors
__global__ void k_dot2(const float* __restrict__ a, const float* __restrict__ b, size_t n, double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        s += (double)a[k] * (double)b[k];
    s = group_sum_d<32>(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        t = group_sum_d<32>(t);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}

__global__ void k_sum_parts(const double* part, int nb, double* out) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) s += part[b];
    s = group_sum_d<32>(s);
    if (threadIdx.x == 0) *out = s;
}

constexpr int kDotBlocks = 296;

// out = a.b in FP64 (device scalar).
void dot_device(fsd_handle* h, const float* a, const float* b, size_t n, double* out) {
    count_launch();
    k_dot2<<<kDotBlocks, 256, 0, h->stream>>>(a, b, n, h->w.dred);
    count_launch();
    k_sum_parts<<<1, 32, 0, h->stream>>>(h->w.dred, kDotBlocks, out);
}

// Lanczos three-term step: w <- (w - beta v_prev - alpha v) and alpha = v.w
__global__ void k_axpby(float* __restrict__ y, const float* __restrict__ x, float a, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        y[k] += a * x[k];
}
__global__ void k_scale(float* __restrict__ y, const float* __restrict__ x, float a, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        y[k] = a * x[k];
}
__global__ void k_lincomb(const float* __restrict__ V, size_t ld, int m, const double* __restrict__ c,
                          float* __restrict__ y, size_t n, float scale) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int i = 0; i < m; ++i) acc += c[i] * (double)V[(size_t)i * ld + k];
        y[k] = (float)(scale * acc);
    }
}

static void vblocks(size_t n, int* b) { *b = (int)std::min<size_t>(4 * 148, (n + 255) / 256); }

// ------------------------------------------------- tridiagonal eigensolver
// Eigen-decomposition of the symmetric tridiagonal matrix (d, e) by the
// implicit QL algorithm with Wilkinson shifts; on return d holds the
// eigenvalues and Z (m x m, row-major, Z[i*m + k] = component i of vector k)
// the eigenvectors.  Returns false if it fails to converge.
bool tridiag_eigen(int m, std::vector<double>& d, std::vector<double> e, std::vector<double>& Z) {
    Z.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i) Z[(size_t)i * m + i] = 1.0;
    e.push_back(0.0);
    for (int l = 0; l < m; ++l) {
        int iter = 0;
        for (;;) {
            int mm = l;
            for (; mm < m - 1; ++mm) {
                const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
                if (fabs(e[mm]) <= 1e-15 * dd) break;
            }
            if (mm == l) break;
            if (++iter > 60) return false;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = mm - 1;
            for (; i >= l; --i) {
                double f = s * e[i], b = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[mm] = 0.0;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < m; ++k) {
                    f = Z[(size_t)k * m + i + 1];
                    Z[(size_t)k * m + i + 1] = s * Z[(size_t)k * m + i] + c * f;
                    Z[(size_t)k * m + i] = c * Z[(size_t)k * m + i] - s * f;
                }
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    return true;
}

// z = f(T) e1 with f = sqrt, T the m x m Lanczos tridiagonal (Helper_Brownian.cu:476-583).
static bool sqrt_T_e1(int m, const std::vector<double>& alpha, const std::vector<double>& beta, std::vector<double>& z) {
    std::vector<double> d(alpha.begin(), alpha.begin() + m), e(beta.begin() + 1, beta.begin() + m), Z;
    if (!tridiag_eigen(m, d, e, Z)) return false;
    z.assign(m, 0.0);
    for (int k = 0; k < m; ++k) {
        if (!(d[k] >= 0.0)) {
            if (d[k] > -1e-12 * fabs(d[m - 1])) d[k] = 0.0;
            else return false;
        }
        const double w = sqrt(d[k]) * Z[k];  // row 0, column k
        for (int i = 0; i < m; ++i) z[i] += Z[(size_t)i * m + k] * w;
    }
    return true;
}

// --------------------------------------------------------------- Lanczos
// y = ||x|| V_m sqrt(T_m) e1 ~ A^1/2 x for the operator `apply` (n = 11N or
// 6N), starting from the carried iteration count *m_io, adding one
// iteration at a time until the relative change of y drops below tol
// (Brownian_FarField.cu:597-808).  The change is measured in the Lanczos
// coordinates, ||z_m - (z_{m-1}, 0)||, which equals the change of y while the
// basis stays orthonormal.  Returns FSD_OK or FSD_ERR_LANCZOS_MAXIT.
int lanczos_sqrt(fsd_handle* h, size_t n, const float* x, float* y, int* m_io, float tol, float scale,
                 const std::function<int(const float*, float*)>& apply, int* iters, float* err_out) {
    Workspace& w = h->w;
    cudaStream_t st = h->stream;
    const int mmax = h->p.lanczos_max;
    float* V = w.lanczos_V;
    int nb;
    vblocks(n, &nb);
    double* hd = w.lz_host;
    // v_1 = x / ||x||
    dot_device(h, x, x, n, w.lz_dot);
    FSD_CHECK_CUDA(cudaMemcpyAsync(hd, w.lz_dot, sizeof(double), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    const double xnorm = sqrt(hd[0]);
    if (!(xnorm > 0.0)) {
        FSD_CHECK_CUDA(cudaMemsetAsync(y, 0, sizeof(float) * n, st));
        if (iters) *iters = 0;
        if (err_out) *err_out = 0.f;
        return FSD_OK;
    }
    count_launch();
    k_scale<<<nb, 256, 0, st>>>(V, x, (float)(1.0 / xnorm), n);
    std::vector<double> alpha, beta(1, 0.0), z, zprev;
    int m = std::max(1, std::min(*m_io, mmax - 2));
    double err = 1.0;
    bool stop = false;
    int k = 0;
    auto step = [&](int j) -> int {
        // w = A v_j - beta_j v_{j-1}; alpha_j = v_j.w; w -= alpha_j v_j; beta_{j+1} = ||w||
        float* vj = V + (size_t)j * n;
        float* wv = V + (size_t)(j + 1) * n;
        int e = apply(vj, wv);
        if (e != FSD_OK) return e;
        ProfRegion pl(h, R_LANCZOS);
        if (j > 0) {
            count_launch();
            count_launch();
            k_axpby<<<nb, 256, 0, st>>>(wv, V + (size_t)(j - 1) * n, (float)(-beta[j]), n);
        }
        dot_device(h, vj, wv, n, w.lz_dot);
        FSD_CHECK_CUDA(cudaMemcpyAsync(hd, w.lz_dot, sizeof(double), cudaMemcpyDeviceToHost, st));
        FSD_CHECK_CUDA(cudaStreamSynchronize(st));
        const double a = hd[0];
        alpha.push_back(a);
        count_launch();
        k_axpby<<<nb, 256, 0, st>>>(wv, vj, (float)(-a), n);
        dot_device(h, wv, wv, n, w.lz_dot);
        FSD_CHECK_CUDA(cudaMemcpyAsync(hd, w.lz_dot, sizeof(double), cudaMemcpyDeviceToHost, st));
        FSD_CHECK_CUDA(cudaStreamSynchronize(st));
        const double b = sqrt(std::max(hd[0], 0.0));
        beta.push_back(b);
        if (b < 1e-8) {
            stop = true;  // invariant subspace (Brownian_FarField.cu:571-579)
        } else {
            count_launch();
            k_scale<<<nb, 256, 0, st>>>(wv, wv, (float)(1.0 / b), n);
        }
        return FSD_OK;
    };
    for (k = 0; k < m && !stop; ++k) {
        int e = step(k);
        if (e != FSD_OK) return e;
    }
    if (!sqrt_T_e1(k, alpha, beta, zprev)) return FSD_ERR_BREAKDOWN;
    z = zprev;
    while (!stop && err > tol && k < mmax - 1) {
        int e = step(k);
        if (e != FSD_OK) return e;
        ++k;
        if (!sqrt_T_e1(k, alpha, beta, z)) return FSD_ERR_BREAKDOWN;
        double dn = 0.0, yn = 0.0;
        for (int i = 0; i < k; ++i) {
            const double d = z[i] - (i < (int)zprev.size() ? zprev[i] : 0.0);
            dn += d * d;
            yn += z[i] * z[i];
        }
        err = yn > 0 ? sqrt(dn / yn) : 0.0;
        zprev = z;
    }
    FSD_CHECK_CUDA(cudaMemcpyAsync(w.lz_dot, z.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
    count_launch();
    k_lincomb<<<nb, 256, 0, st>>>(V, n, k, w.lz_dot, y, n, (float)(xnorm * scale));
    FSD_CHECK_CUDA(cudaGetLastError());
    *m_io = std::max(1, k - 1);
    if (iters) *iters = k;
    if (err_out) *err_out = (float)(stop ? 0.0 : err);
    return (err > tol && !stop) ? FSD_ERR_LANCZOS_MAXIT : FSD_OK;
}

// ------------------------------------------------------------- far field
int brownian_farfield(fsd_handle* h, const float4* pos, uint32_t step, float* out11) {
    Workspace& w = h->w;
    const int N = h->p.N;
    const size_t n = 11 * (size_t)N;
    const GridParams& g = h->g;
    const float T = h->p.T, dt = h->p.dt;
    const float quadW = g.hx * g.hy * g.hz;
    const float fac = sqrtf(T / dt / quadW);
    const int G = g.Nx * g.Ny * g.Nz;
    // Wave space: random spectrum, inverse FFT, contraction.
    {
        ProfRegion prw(h, R_BROWNIAN_WAVE);
    count_launch();
    k_noise_spectrum<<<(G + 255) / 256, 256, 0, h->stream>>>(w.grid, w.gridk, g.Nx, g.Ny, g.Nz, fac, h->seed_hashed,
                                                             step, kStreamFFWave);
    mobility_wave_from_spectrum(h, pos);
    // Combine into generalized layout (wave part only): needs f4/c4 unused.
    mobility_combine(h, pos, nullptr, w.lz_c, true, false, nullptr);
    }
    // Real space: Lanczos square root of M_real on an 11N normal vector.
    float* psi = w.lz_a;
    gaussian(h, psi, n, step, kStreamFFReal, 1.0f);
    auto apply = [&](const float* v, float* o) { return mobility_apply(h, pos, v, o, 2, nullptr, false); };
    int it = 0;
    float err = 0.f;
    const int st = lanczos_sqrt(h, n, psi, w.lz_b, &h->m_lanczos_ff, h->p.lanczos_tol, sqrtf(2.0f * T / dt), apply,
                                &it, &err);
    h->info.lanczos_ff_iters = it;
    h->info.lanczos_ff_err = err;
    if (st != FSD_OK && st != FSD_ERR_LANCZOS_MAXIT) return st;
    // out = wave + real
    count_launch();
    k_scale<<<(int)std::min<size_t>(4 * 148, (n + 255) / 256), 256, 0, h->stream>>>(out11, w.lz_c, 1.0f, n);
    count_launch();
    k_axpby<<<(int)std::min<size_t>(4 * 148, (n + 255) / 256), 256, 0, h->stream>>>(out11, w.lz_b, 1.0f, n);
    FSD_CHECK_CUDA(cudaGetLastError());
    return st;
}

// ------------------------------------------------------------ near field
int brownian_nearfield(fsd_handle* h, const float4* pos, uint32_t step, float* out6) {
    Workspace& w = h->w;
    const int N = h->p.N;
    const size_t n = 6 * (size_t)N;
    float* psi = w.lz_a;
    gaussian(h, psi, n, step, kStreamNF, 1.0f);
    auto apply = [&](const float* v, float* o) {
        lub_rfu(h, pos, v, o, nullptr);
        return FSD_OK;
    };
    int it = 0;
    float err = 0.f;
    const float s = sqrtf(2.0f * h->p.T / h->p.dt);
    const int st = lanczos_sqrt(h, n, psi, out6, &h->m_lanczos_nf, h->p.lanczos_tol, s, apply, &it, &err);
    h->info.lanczos_nf_iters = it;
    h->info.lanczos_nf_err = err;
    return st;
}

// ------------------------------------------------------------------- drift
__global__ void k_displace(const float4* __restrict__ pos, float4* __restrict__ out, const float* __restrict__ psi,
                           int N, Box b, float d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 p = pos[i];
    float3 x = make_float3(p.x + psi[6 * i] * d, p.y + psi[6 * i + 1] * d, p.z + psi[6 * i + 2] * d);
    int3 img = make_int3(0, 0, 0);
    wrap_position(x, img, b);
    out[i] = make_float4(x.x, x.y, x.z, p.w);
}

__global__ void k_rfd_rhs(float* rhs, const float* psi, int N) {
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k < 17 * (size_t)N) rhs[k] = (k >= 11 * (size_t)N) ? -psi[k - 11 * (size_t)N] : 0.0f;
}

__global__ void k_rfd_finish(float* drift, const float* up, const float* um, int N, float fac) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 6 * N) drift[k] = fac * up[k] - fac * um[k];
}

// U_drift = (kT/eps) (U(x + eps psi/2) - U(x - eps psi/2)) with A(x') U = (0; -psi),
// reusing the neighbour list and preconditioner built at x (Integrator.cu:549-718).
int rfd_drift(fsd_handle* h, const float4* pos, uint32_t step, float* drift6) {
    Workspace& w = h->w;
    const int N = h->p.N;
    const float eps = h->p.rfd_epsilon;
    gaussian(h, w.psi, 6 * (size_t)N, step, kStreamRFD, 1.0f);
    count_launch();
    k_rfd_rhs<<<(17 * N + 255) / 256, 256, 0, h->stream>>>(w.rfd_rhs, w.psi, N);
    FSD_CHECK_CUDA(cudaMemsetAsync(w.rfd_sol, 0, sizeof(float) * 17 * N, h->stream));
    count_launch();
    k_displace<<<(N + 127) / 128, 128, 0, h->stream>>>(pos, w.pos_prime, w.psi, N, h->box, eps / 2.0f);
    int it = 0;
    float res = 0.f;
    int st = saddle_solve(h, w.pos_prime, w.rfd_rhs, w.rfd_sol, h->p.solver_tol, &it, &res);
    h->info.gmres_iters[0] = it;
    h->info.gmres_resid[0] = res;
    // A solve that stops above its tolerance keeps its best solution, as the
    // reference continues after its non-convergence message (Solvers.cu:121).
    int status = FSD_OK;
    if (st == FSD_ERR_GMRES_MAXIT) status = st;
    else if (st != FSD_OK) return st;
    FSD_CHECK_CUDA(cudaMemcpyAsync(w.vel, w.rfd_sol + 11 * N, sizeof(float) * 6 * N, cudaMemcpyDeviceToDevice,
                                   h->stream));
    count_launch();
    k_displace<<<(N + 127) / 128, 128, 0, h->stream>>>(pos, w.pos_prime, w.psi, N, h->box, -eps / 2.0f);
    st = saddle_solve(h, w.pos_prime, w.rfd_rhs, w.rfd_sol, h->p.solver_tol, &it, &res);
    h->info.gmres_iters[1] = it;
    h->info.gmres_resid[1] = res;
    if (st == FSD_ERR_GMRES_MAXIT) status = st;
    else if (st != FSD_OK) return st;
    count_launch();
    k_rfd_finish<<<(6 * N + 255) / 256, 256, 0, h->stream>>>(drift6, w.vel, w.rfd_sol + 11 * N, N, h->p.T / eps);
    // Positions used by the mobility bins must be rebinned for x on the next matvec.
    FSD_CHECK_CUDA(cudaGetLastError());
    return status;
}

}  // namespace fsd
