// Far-field grand mobility by the Positively Split Ewald method
// (Mobility.cu, Helper_Mobility.cu of the reference):
//
//   wave space:  spread F and couplet C to 11 real grids with Gaussians of
//                support P^3, 3D FFT, scale by the Hasimoto/RPY Green's
//                function, inverse FFT, contract back to particles;
//   real space:  tabulated pair sum within ewald_cut plus the self term.
//
// B200 layout choices:
//   * the 11 real grids are carried as 6 complex grids (two real grids per
//     complex grid: F_x+iF_y, C_xx+iC_xy, C_xz+iC_yx, C_yy+iC_yz, C_zx+iC_zy,
//     F_z), so forward and inverse transforms are 6 complex FFTs each instead
//     of the reference's 11 + 11 (the grids are real before the forward
//     transform and only real parts are read after the inverse one);
//   * spreading is a per-tile gather over particles binned by stencil origin,
//     so every grid node is written exactly once with a fixed summation order
//     (no atomics, deterministic);
//   * the FFT is a shared-memory mixed-radix Stockham transform along each
//     axis over batches of lines; the whole 72^3 working set (18 MB) stays in
//     the 126 MB L2.
#include <algorithm>
#include <cmath>

#include <array>
#include <functional>
#include <map>
#include <mutex>

#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_profile.h"

namespace fsd {

namespace {
constexpr float kPiRef = 3.1415926536f;  // the reference's pi literal
}

// ------------------------------------------------------------------ FFT plan
FFTPlan make_fft_plan(int n) {
    FFTPlan p{};
    p.n = n;
    int m = n, k = 0;
    const int radices[] = {8, 5, 4, 3, 2};
    while (m > 1) {
        bool found = false;
        for (int r : radices) {
            if (m % r == 0) {
                p.radix[k++] = r;
                m /= r;
                found = true;
                break;
            }
        }
        if (!found) {
            p.nst = -1;
            return p;
        }
    }
    p.nst = k;
    return p;
}

// Twiddle tables w_n^m = exp(-2 pi i m / n), m in [0, n), for the three axes,
// computed in double on the host.
void fill_twiddles(fsd_handle* h) {
    const int ns[3] = {h->g.Nx, h->g.Ny, h->g.Nz};
    std::vector<float2> tw(ns[0] + ns[1] + ns[2]);
    int off = 0;
    for (int a = 0; a < 3; ++a) {
        for (int m = 0; m < ns[a]; ++m) {
            const double ang = -2.0 * M_PI * (double)m / (double)ns[a];
            tw[off + m] = make_float2((float)cos(ang), (float)sin(ang));
        }
        off += ns[a];
    }
    cudaMemcpyAsync(h->w.twiddle, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice, h->stream);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// Radix-P DFT of y[0..P) in place with the roots w_P^m = exp(-2 pi i m / P)
// as constants (conjugated for the inverse).
// cos and sin of -2 pi m / P for the radices used (m < P); folded to
// constants once the DFT loops are unrolled.
// Radix 9 uses cos and sin of 2 pi m / 9, m = 1..4, mirrored.
__host__ __device__ constexpr float root9_c(int m) {
    return (m == 0) ? 1.0f
         : (m == 1 || m == 8) ? 0.76604444311897804f
         : (m == 2 || m == 7) ? 0.17364817766693035f
         : (m == 3 || m == 6) ? -0.5f
         : -0.93969262078590838f;
}
__host__ __device__ constexpr float root9_s(int m) {
    return (m == 0) ? 0.0f
         : (m == 1) ? -0.64278760968653933f : (m == 8) ? 0.64278760968653933f
         : (m == 2) ? -0.98480775301220806f : (m == 7) ? 0.98480775301220806f
         : (m == 3) ? -0.86602540378443865f : (m == 6) ? 0.86602540378443865f
         : (m == 4) ? -0.34202014332566873f : 0.34202014332566873f;
}
__host__ __device__ constexpr float root_c(int P, int m) {
    return P == 9 ? root9_c(m)
         : P == 2 ? (m == 0 ? 1.0f : -1.0f)
         : P == 3 ? (m == 0 ? 1.0f : -0.5f)
         : P == 4 ? (m == 0 ? 1.0f : (m == 2 ? -1.0f : 0.0f))
         : P == 5 ? (m == 0 ? 1.0f : (m == 1 || m == 4) ? 0.30901699437494742f : -0.80901699437494742f)
         : /* 8 */ (m == 0 ? 1.0f : m == 4 ? -1.0f : (m == 2 || m == 6) ? 0.0f
                    : (m == 1 || m == 7) ? 0.70710678118654752f : -0.70710678118654752f);
}
__host__ __device__ constexpr float root_s(int P, int m) {
    return P == 9 ? root9_s(m)
         : P == 2 ? 0.0f
         : P == 3 ? (m == 0 ? 0.0f : m == 1 ? -0.86602540378443865f : 0.86602540378443865f)
         : P == 4 ? (m == 1 ? -1.0f : m == 3 ? 1.0f : 0.0f)
         : P == 5 ? (m == 0 ? 0.0f : m == 1 ? -0.95105651629515357f : m == 2 ? -0.58778525229247313f
                    : m == 3 ? 0.58778525229247313f : 0.95105651629515357f)
         : /* 8 */ (m == 0 || m == 4 ? 0.0f : m == 2 ? -1.0f : m == 6 ? 1.0f
                    : (m == 1 || m == 3) ? -0.70710678118654752f : 0.70710678118654752f);
}

template <int P>
__device__ __forceinline__ void small_dft(float2* y, bool inv) {
    const float sg = inv ? -1.0f : 1.0f;
    float2 z[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        float2 acc = y[0];
#pragma unroll
        for (int s = 1; s < P; ++s) {
            const int m = (j * s) % P;
            const float wc = root_c(P, m), ws = sg * root_s(P, m);
            acc.x += y[s].x * wc - y[s].y * ws;
            acc.y += y[s].x * ws + y[s].y * wc;
        }
        z[j] = acc;
    }
#pragma unroll
    for (int j = 0; j < P; ++j) y[j] = z[j];
}

// floor(a / d) for a < 2^20 and 1 <= d <= 2^12 from a float reciprocal: the
// true quotient plus 0.5/d stays at least 0.5/d away from an integer, more
// than the rounding error of the product (a/d * 2^-22 < 0.25/d).
__device__ __forceinline__ int qdiv(int a, float inv_d, float half_inv) {
    return (int)__fmaf_rn((float)a, inv_d, half_inv);
}

// One Stockham stage of radix P over nlines lines of length n; Ls = product of
// the radices before it.  The twiddle index j1 * s * r is below n (j1 < Ls,
// r = n / (Ls P), s < P), so no reduction is needed.
template <int P>
__device__ __forceinline__ void stockham_stage(const float2* in, float2* out, int nlines, int n, int Ls,
                                               const float2* tw, bool inv) {
    const int L = Ls * P, r = n / L, nb = n / P;
    const float inv_nb = 1.0f / (float)nb, h_nb = 0.5f / (float)nb;
    const float inv_r = 1.0f / (float)r, h_r = 0.5f / (float)r;
    const int total = nlines * nb;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        const int line = qdiv(w, inv_nb, h_nb), bf = w - line * nb;
        const int j1 = qdiv(bf, inv_r, h_r), k = bf - j1 * r;
        const float2* X = in + line * n;
        float2* Y = out + line * n;
        float2 y[P];
#pragma unroll
        for (int s = 0; s < P; ++s) {
            float2 v = X[k + s * r + r * P * j1];
            if (s > 0 && j1 > 0) {
                float2 t = tw[j1 * s * r];
                if (inv) t.y = -t.y;
                v = cmul(v, t);
            }
            y[s] = v;
        }
        small_dft<P>(y, inv);
#pragma unroll
        for (int j2 = 0; j2 < P; ++j2) Y[k + r * (j1 + Ls * j2)] = y[j2];
    }
}

// Transforms nlines lines of length n held in a (ping-pong with b); returns
// the buffer holding the result.
__device__ float2* fft_lines(float2* a, float2* b, int nlines, const FFTPlan& pl, const float2* tw, bool inv) {
    float2* in = a;
    float2* out = b;
    int Ls = 1;
    for (int q = 0; q < pl.nst; ++q) {
        const int p = pl.radix[q];
        switch (p) {
            case 2: stockham_stage<2>(in, out, nlines, pl.n, Ls, tw, inv); break;
            case 3: stockham_stage<3>(in, out, nlines, pl.n, Ls, tw, inv); break;
            case 4: stockham_stage<4>(in, out, nlines, pl.n, Ls, tw, inv); break;
            case 5: stockham_stage<5>(in, out, nlines, pl.n, Ls, tw, inv); break;
            default: stockham_stage<8>(in, out, nlines, pl.n, Ls, tw, inv); break;
        }
        __syncthreads();
        float2* t = in;
        in = out;
        out = t;
        Ls *= p;
    }
    return in;
}

// One axis of the 3D transform for all 6 packed grids.  axis 2 (z): batches of
// B contiguous lines; axes 1 (y) and 0 (x): lines grouped by B consecutive z.
__global__ void __launch_bounds__(256, 4) k_fft_axis(float2* __restrict__ data, int Nx, int Ny, int Nz, int axis, int B, FFTPlan pl,
                           const float2* __restrict__ tw_global, bool inv, int ngrids) {
    extern __shared__ float2 smem[];
    const int n = pl.n;
    float2* tw = smem;
    float2* a = smem + n;
    float2* b = a + B * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_global[i];
    const size_t G = (size_t)Nx * Ny * Nz;
    size_t base;
    int nl, es, ls;  // valid lines, element stride, line stride
    if (axis == 2) {
        const size_t lines_total = (size_t)ngrids * Nx * Ny;
        const size_t l0 = (size_t)blockIdx.x * B;
        nl = (int)min((size_t)B, lines_total - l0);
        const size_t g = l0 / ((size_t)Nx * Ny);
        const size_t xy = l0 % ((size_t)Nx * Ny);
        base = g * G + xy * Nz;  // lines of one batch never straddle grids: (Nx*Ny) % B handled by host
        es = 1;
        ls = Nz;
    } else {
        const int nch = (Nz + B - 1) / B;
        const int outer = (axis == 1) ? Nx : Ny;
        int bid = blockIdx.x;
        const int ch = bid % nch;
        bid /= nch;
        const int o = bid % outer;
        const int g = bid / outer;
        const int z0 = ch * B;
        nl = min(B, Nz - z0);
        es = (axis == 1) ? Nz : Ny * Nz;
        base = (size_t)g * G + (axis == 1 ? (size_t)o * Ny * Nz : (size_t)o * Nz) + z0;
        ls = 1;
    }
    const int tot = nl * n;
    if (axis == 2) {
        for (int i = threadIdx.x; i < tot; i += blockDim.x) {
            const int line = i / n, t = i - line * n;
            a[line * n + t] = data[base + (size_t)line * ls + t];
        }
    } else {
        for (int i = threadIdx.x; i < tot; i += blockDim.x) {
            const int t = i / nl, line = i - t * nl;
            a[line * n + t] = data[base + (size_t)t * es + line];
        }
    }
    __syncthreads();
    float2* res = fft_lines(a, b, nl, pl, tw, inv);
    if (axis == 2) {
        for (int i = threadIdx.x; i < tot; i += blockDim.x) {
            const int line = i / n, t = i - line * n;
            data[base + (size_t)line * ls + t] = res[line * n + t];
        }
    } else {
        for (int i = threadIdx.x; i < tot; i += blockDim.x) {
            const int t = i / nl, line = i - t * nl;
            data[base + (size_t)t * es + line] = res[line * n + t];
        }
    }
}

// y and z passes of one (grid, x) plane in a single kernel, for Ny = Nz = N =
// N1 * N2.  The N x N plane (contiguous in global memory, z fastest) sits in
// shared memory with row stride N + 1.  Each length-N line is transformed in
// two in-place stages (Cooley-Tukey, N = N1 N2): the N2-point DFTs over the
// stride-N1 subsequences with the twiddles w_N^(n1 k2), then the N1-point DFTs
// over contiguous runs of N1, each writing its outputs into the slots it
// read.  Coefficient k = k2 + N2 k1 of a line therefore ends at slot
// k1 + N1 k2; the store undoes that order on both axes.  Forward: z lines,
// then y lines; inverse: y, then z (the order of the separate passes).
template <int N1, int N2>
__device__ __forceinline__ int plane_slot(int k) {
    return k / N2 + N1 * (k % N2);
}

template <int N1, int N2>
__device__ __forceinline__ void plane_lines(float2* pl, const float2* tw, bool rows, bool inv) {
    constexpr int N = N1 * N2, RS = N + 1;
    // element i of line l: rows (z lines) at l * RS + i, columns (y lines) at i * RS + l
    const int es = rows ? 1 : RS, ls = rows ? RS : 1;
    for (int t = threadIdx.x; t < N * N1; t += blockDim.x) {
        const int l = t % N, n1 = t / N;  // consecutive threads: consecutive lines
        float2* L = pl + l * ls + n1 * es;
        float2 y[N2];
#pragma unroll
        for (int q = 0; q < N2; ++q) y[q] = L[q * N1 * es];
        small_dft<N2>(y, inv);
#pragma unroll
        for (int q = 0; q < N2; ++q) {
            float2 w = tw[n1 * q];
            if (inv) w.y = -w.y;
            L[q * N1 * es] = q == 0 ? y[0] : cmul(y[q], w);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < N * N2; t += blockDim.x) {
        const int l = t % N, k2 = t / N;
        float2* L = pl + l * ls + k2 * N1 * es;
        float2 y[N1];
#pragma unroll
        for (int q = 0; q < N1; ++q) y[q] = L[q * es];
        small_dft<N1>(y, inv);
#pragma unroll
        for (int q = 0; q < N1; ++q) L[q * es] = y[q];
    }
    __syncthreads();
}

template <int N1, int N2>
__global__ void __launch_bounds__(256) k_fft_yz(float2* __restrict__ data, int Nx, const float2* __restrict__ tw_global,
                                                bool inv) {
    constexpr int N = N1 * N2, RS = N + 1;
    extern __shared__ float2 smem[];
    float2* tw = smem;
    float2* pl = smem + N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_global[i];
    const size_t base = (size_t)blockIdx.x * N * N;  // blocks are (grid, x) planes in memory order
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        const int y = e / N, z = e - y * N;
        pl[y * RS + z] = data[base + e];
    }
    __syncthreads();
    if (!inv) {
        plane_lines<N1, N2>(pl, tw, true, false);
        plane_lines<N1, N2>(pl, tw, false, false);
    } else {
        plane_lines<N1, N2>(pl, tw, false, true);
        plane_lines<N1, N2>(pl, tw, true, true);
    }
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        const int y = e / N, z = e - y * N;
        data[base + e] = pl[plane_slot<N1, N2>(y) * RS + plane_slot<N1, N2>(z)];
    }
}

// Launches the plane kernel when Ny = Nz has a specialisation; false otherwise.
static bool fft_yz(fsd_handle* h, bool inv, int ngrids, const float2* twyz) {
    const int Nx = h->g.Nx, N = h->g.Ny;
    if (h->g.Nz != N) return false;
    const size_t shm = sizeof(float2) * ((size_t)N + (size_t)N * (N + 1));
    const int nblocks = ngrids * Nx;
    auto go = [&](auto kern) {
        if (!smem_limit_ok((const void*)kern, shm, "k_fft_yz shared memory")) return;
        count_launch();
        kern<<<nblocks, 256, shm, h->stream>>>(h->w.grid, Nx, twyz, inv);
    };
    switch (N) {
        case 72: go(k_fft_yz<8, 9>); return true;
        case 36: go(k_fft_yz<4, 9>); return true;
        case 27: go(k_fft_yz<3, 9>); return true;
        default: return false;
    }
}

static int fft_batch_z(int Nx, int Ny, int Nz) {
    // Batches must not straddle two grids: pick B dividing Nx*Ny.
    int B = std::max(1, 2048 / Nz);
    while (B > 1 && (Nx * Ny) % B != 0) --B;
    return B;
}

static void fft3d(fsd_handle* h, bool inv, int ngrids, bool skip_x = false) {
    const int Nx = h->g.Nx, Ny = h->g.Ny, Nz = h->g.Nz;
    const FFTPlan px = make_fft_plan(Nx), py = make_fft_plan(Ny), pz = make_fft_plan(Nz);
    const float2* twx = h->w.twiddle;
    const float2* twy = twx + Nx;
    const float2* twz = twy + Ny;
    // x and y passes: lines of consecutive z, B of them per block; a divisor
    // of Nz avoids a partial last chunk.
    int Bxy = 16;
    for (int d = 32; d >= 8; --d)
        if (Nz % d == 0) {
            Bxy = d;
            break;
        }
    int Bz = fft_batch_z(Nx, Ny, Nz);
    if (h->tune.set && h->tune.Bxy > 0) {
        Bxy = h->tune.Bxy;
        Bz = h->tune.Bz;
    }
    auto launch = [&](int axis) {
        const FFTPlan& pl = axis == 0 ? px : (axis == 1 ? py : pz);
        const float2* tw = axis == 0 ? twx : (axis == 1 ? twy : twz);
        const int B = axis == 2 ? Bz : Bxy;
        int nblocks;
        if (axis == 2)
            nblocks = (int)(((size_t)ngrids * Nx * Ny + B - 1) / B);
        else
            nblocks = ngrids * (axis == 1 ? Nx : Ny) * ((Nz + B - 1) / B);
        const size_t shm = sizeof(float2) * ((size_t)pl.n + 2 * (size_t)B * pl.n);
        if (!smem_limit_ok((const void*)k_fft_axis, shm, "k_fft_axis shared memory")) return;
        count_launch();
        k_fft_axis<<<nblocks, 256, shm, h->stream>>>(h->w.grid, Nx, Ny, Nz, axis, B, pl, tw, inv, ngrids);
    };
    // y and z twiddles coincide when Ny = Nz (both tables are exp(-2 pi i m / N)).
    if (!inv) {
        if (!fft_yz(h, false, ngrids, twz)) {
            launch(2);
            launch(1);
        }
        if (!skip_x) launch(0);
    } else {
        if (!skip_x) launch(0);
        if (!fft_yz(h, true, ngrids, twz)) {
            launch(1);
            launch(2);
        }
    }
}

// ------------------------------------------------------------- wave vectors
// Wave vector and Green's scale per grid point (Mobility_SetGridk_kernel,
// Helper_Mobility.cu:351-410), keeping its mixed float/double arithmetic.
__global__ void k_gridk(float4* gridk, int Nx, int Ny, int Nz, Box b, float xi, float eta, double two_pi) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int G = Nx * Ny * Nz;
    if (tid >= G) return;
    const int i = tid / (Ny * Nz);
    const int j = (tid - i * Ny * Nz) / Nz;
    const int k = tid % Nz;
    float4 v;
    v.x = (float)((i < (Nx + 1) / 2) ? i : i - Nx);
    v.y = ((float)((j < (Ny + 1) / 2) ? j : j - Ny) - b.xy * v.x * b.Ly / b.Lx) / b.Ly;
    v.x = v.x / b.Lx;
    v.z = (float)((k < (Nz + 1) / 2) ? k : k - Nz) / b.Lz;
    v.x = (float)(v.x * two_pi);
    v.y = (float)(v.y * two_pi);
    v.z = (float)(v.z * two_pi);
    const float k2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const float xisq = xi * xi;
    if (tid == 0) {
        v.w = 0.0f;
    } else {
        const float e = (float)(-(1 - eta) * (double)k2 / 4.0 / (double)xisq);
        v.w = (float)(6.0 * 3.1415926536 * (1.0 + (double)k2 / 4.0 / (double)xisq) * (double)expf(e) / (double)k2 /
                      (double)G);
    }
    gridk[tid] = v;
}

void mobility_set_gridk(fsd_handle* h) {
    const int G = h->g.Nx * h->g.Ny * h->g.Nz;
    const double two_pi = h->p.kgrid_pi_ref ? 2.0 * 3.1416926536 : 2.0 * M_PI;
    count_launch();
    k_gridk<<<(G + 255) / 256, 256, 0, h->stream>>>(h->w.gridk, h->g.Nx, h->g.Ny, h->g.Nz, h->box, h->p.xi, h->g.eta,
                                                    two_pi);
}

// ---------------------------------------------------------------- Green step
// Spectra order: X Y Z XX XY XZ YX YY YZ ZX ZY (force then couplet / velocity
// then velocity gradient), as Mobility_WaveSpace_Green_kernel (Mobility.cu:315).
// sgn = +1 applies the operator at wave vector tk; sgn = -1 applies the
// operator with its imaginary-unit couplings conjugated (used to average with
// the mirror point on Nyquist planes).
__device__ __forceinline__ void green_apply(const float4 tk, const float2* f, float2* o, float sgn) {
    const float2 fX = f[0], fY = f[1], fZ = f[2];
    const float2 cXX = f[3], cXY = f[4], cXZ = f[5], cYX = f[6], cYY = f[7], cYZ = f[8], cZX = f[9], cZY = f[10];
    const float2 cZZ = make_float2(-(cXX.x + cYY.x), -(cXX.y + cYY.y));
    const float ksq = tk.x * tk.x + tk.y * tk.y + tk.z * tk.z;
    const float k = sqrtf(ksq);
    const float2 kdF = make_float2((tk.x * fX.x + tk.y * fY.x + tk.z * fZ.x) / ksq,
                                   (tk.x * fX.y + tk.y * fY.y + tk.z * fZ.y) / ksq);
    const float2 Cdkx = make_float2(cXX.x * tk.x + cXY.x * tk.y + cXZ.x * tk.z, cXX.y * tk.x + cXY.y * tk.y + cXZ.y * tk.z);
    const float2 Cdky = make_float2(cYX.x * tk.x + cYY.x * tk.y + cYZ.x * tk.z, cYX.y * tk.x + cYY.y * tk.y + cYZ.y * tk.z);
    const float2 Cdkz = make_float2(cZX.x * tk.x + cZY.x * tk.y + cZZ.x * tk.z, cZX.y * tk.x + cZY.y * tk.y + cZZ.y * tk.z);
    const float2 kdcdk = make_float2((Cdkx.x * tk.x + Cdky.x * tk.y + Cdkz.x * tk.z) / ksq,
                                     (Cdkx.y * tk.x + Cdky.y * tk.y + Cdkz.y * tk.z) / ksq);
    const float sk = sinf(k), ck = cosf(k);
    const float j0 = sk / k;
    const float j1k = (sk - k * ck) / (ksq * k);
    // UF: (I - kk) F, real scale.
    const float Buf = tk.w * j0 * j0;
    o[0] = make_float2((fX.x - tk.x * kdF.x) * Buf, (fX.y - tk.x * kdF.y) * Buf);
    o[1] = make_float2((fY.x - tk.y * kdF.x) * Buf, (fY.y - tk.y * kdF.y) * Buf);
    o[2] = make_float2((fZ.x - tk.z * kdF.x) * Buf, (fZ.y - tk.z * kdF.y) * Buf);
    // UC: imaginary scale.
    const float Buc = sgn * (float)((double)(-tk.w * j0) * (3.0 * (double)(sk - k * ck) / (double)(ksq * k)));
    o[0].x += -(Cdkx.y - tk.x * kdcdk.y) * Buc;
    o[1].x += -(Cdky.y - tk.y * kdcdk.y) * Buc;
    o[2].x += -(Cdkz.y - tk.z * kdcdk.y) * Buc;
    o[0].y += (Cdkx.x - tk.x * kdcdk.x) * Buc;
    o[1].y += (Cdky.x - tk.y * kdcdk.x) * Buc;
    o[2].y += (Cdkz.x - tk.z * kdcdk.x) * Buc;
    // DF: imaginary scale, D_ab = i B (F_a k_b - k_a k_b k.F/k^2).
    const float Bdf = sgn * (float)((double)(tk.w * j0) * (3.0 * (double)(sk - k * ck) / (double)(ksq * k)));
    const float fa[3][2] = {{fX.x, fX.y}, {fY.x, fY.y}, {fZ.x, fZ.y}};
    const float kv[3] = {tk.x, tk.y, tk.z};
    const int ia[8] = {0, 0, 0, 1, 1, 1, 2, 2};
    const int ib[8] = {0, 1, 2, 0, 1, 2, 0, 1};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float kk = kv[ia[c]] * kv[ib[c]];
        const float Fkr = fa[ia[c]][0] * kv[ib[c]], Fki = fa[ia[c]][1] * kv[ib[c]];
        o[3 + c] = make_float2(-(Fki - kk * kdF.y) * Bdf, (Fkr - kk * kdF.x) * Bdf);
    }
    // DC: real scale.
    const float Bdc = (float)((double)tk.w * (-1.0) * (-9.0) * (double)j1k * (double)j1k);
    const float2 Cdk[3] = {Cdkx, Cdky, Cdkz};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float kk = kv[ia[c]] * kv[ib[c]];
        o[3 + c].x += (Cdk[ia[c]].x * kv[ib[c]] - kk * kdcdk.x) * Bdc;
        o[3 + c].y += (Cdk[ia[c]].y * kv[ib[c]] - kk * kdcdk.y) * Bdc;
    }
}

// Packed pair p holds spectra (packA(p), packB(p)); compile-time so that the
// unrolled loops keep the spectra in registers.
__host__ __device__ constexpr int packA(int p) { return p == 0 ? 0 : p == 1 ? 3 : p == 2 ? 5 : p == 3 ? 7 : p == 4 ? 9 : 2; }
__host__ __device__ constexpr int packB(int p) { return p == 0 ? 1 : p == 1 ? 4 : p == 2 ? 6 : p == 3 ? 8 : p == 4 ? 10 : -1; }

// Forward x-pass, Green's function and inverse x-pass in one kernel.  A block
// holds, for all 6 packed grids, a set of x-lines closed under the mirror map
// (y, z) -> (-y, -z), so both points of every mirror pair {k, -k} are in
// shared memory.  Blocks [0, Ny * nzc): line y with the z-run
// {1 + c B, ..} inside [1, ceil(Nz / 2)) and the mirrored lines (-y, -z);
// then the planes z = 0 (and z = Nz / 2 for even Nz), pairing y with -y.
// Every line lies in exactly one block.

// Line set of fused x-pass block `bid`: ly/lz of each line and its mirror
// line; returns (lines, primary lines).
__device__ __forceinline__ int2 x_green_lines(int bid, int Ny, int Nz, int B, int nzc, int* ly, int* lz, int* lmir) {
    int nl = 0, np = 0;
    if (bid < Ny * nzc) {
        const int y = bid / nzc, c = bid % nzc;
        const int h = (Nz + 1) / 2;
        const int z0 = 1 + c * B, z1 = min(h, z0 + B);
        const int ym = (Ny - y) % Ny;
        const int cnt = z1 - z0;
        for (int k = 0; k < cnt; ++k) {
            ly[k] = y;
            lz[k] = z0 + k;
            lmir[k] = cnt + k;
            ly[cnt + k] = ym;
            lz[cnt + k] = Nz - (z0 + k);
            lmir[cnt + k] = k;
        }
        nl = 2 * cnt;
        np = cnt;
    } else {
        const int pb = bid - Ny * nzc;
        const int ny_half = Ny / 2 + 1;  // y in [0, Ny/2]
        const int zplane = (pb < ny_half) ? 0 : Nz / 2;
        const int y = (pb < ny_half) ? pb : pb - ny_half;
        const int ym = (Ny - y) % Ny;
        ly[0] = y;
        lz[0] = zplane;
        if (ym != y) {
            ly[1] = ym;
            lz[1] = zplane;
            lmir[0] = 1;
            lmir[1] = 0;
            nl = 2;
        } else {
            lmir[0] = 0;
            nl = 1;
        }
        np = 1;
    }
    return make_int2(nl, np);
}

// Green's function on the mirror pairs {k, -k} of the spectra held in shared
// memory: line q (grid-major, q = p * nl + l) has row stride ls, and
// coefficient x of a line sits at slot(x).  Each pair unpacks the 11 spectra
// of the real grids from the 6 packed complex ones (A = (C(k) + conj C(m)) / 2,
// B = -i (C(k) - conj C(m)) / 2), applies the Green's function (averaged with
// the mirror operator where the mirror wave vector is not -k, i.e. on Nyquist
// planes, which reproduces the real part the reference keeps after its
// complex inverse transform) and repacks (C(k) = A + i B, C(m) = conj A +
// i conj B).  The smaller global index represents the pair; k = 0 is zeroed.
template <class Slot>
__device__ __forceinline__ void x_green_pairs(float2* res, int nl, int np, int ls, Slot slot, const int* ly,
                                              const int* lz, const int* lmir, const float4* __restrict__ gridk,
                                              int Nx, int Ny, int Nz) {
    const int n = Nx;
    for (int t = threadIdx.x; t < np * n; t += blockDim.x) {
        const int l = t / n, x = t - l * n;
        const int lm = lmir[l];
        const int xm = (Nx - x) % Nx;
        if (lm == l && xm < x) continue;  // self-mirror line: each pair once
        size_t idx = ((size_t)x * Ny + ly[l]) * Nz + lz[l];
        size_t m = ((size_t)xm * Ny + ly[lm]) * Nz + lz[lm];
        int sl = l, sx = x, ml = lm, mx = xm;
        if (m < idx) {  // the smaller global index represents the pair
            const size_t tmp = idx;
            idx = m;
            m = tmp;
            sl = lm;
            sx = xm;
            ml = l;
            mx = x;
        }
        const int ps = slot(sx), pm = slot(mx);
        float2 ck[6], cm[6], f[11], o[11];
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            ck[p] = res[(size_t)(p * nl + sl) * ls + ps];
            cm[p] = res[(size_t)(p * nl + ml) * ls + pm];
        }
        if (idx == 0) {
#pragma unroll
            for (int p = 0; p < 6; ++p) res[(size_t)(p * nl + sl) * ls + ps] = make_float2(0.f, 0.f);
            continue;
        }
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            const float2 A = make_float2(0.5f * (ck[p].x + cm[p].x), 0.5f * (ck[p].y - cm[p].y));
            const float2 Bv = make_float2(0.5f * (ck[p].y + cm[p].y), -0.5f * (ck[p].x - cm[p].x));
            f[packA(p)] = A;
            if (packB(p) >= 0) f[packB(p)] = Bv;
        }
        const int i = (int)(idx / ((size_t)Ny * Nz)), j = (int)((idx / Nz) % Ny), k = (int)(idx % Nz);
        green_apply(gridk[idx], f, o, 1.0f);
        if ((2 * i == Nx) || (2 * j == Ny) || (2 * k == Nz)) {
            float2 o2[11];
            green_apply(gridk[m], f, o2, -1.0f);
#pragma unroll
            for (int c = 0; c < 11; ++c) o[c] = make_float2(0.5f * (o[c].x + o2[c].x), 0.5f * (o[c].y + o2[c].y));
        }
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            const float2 A = o[packA(p)];
            const float2 Bv = (packB(p) >= 0) ? o[packB(p)] : make_float2(0.f, 0.f);
            res[(size_t)(p * nl + sl) * ls + ps] = make_float2(A.x - Bv.y, A.y + Bv.x);
            if (m != idx) res[(size_t)(p * nl + ml) * ls + pm] = make_float2(A.x + Bv.y, -A.y + Bv.x);
        }
    }
}

struct IdentitySlot {
    __device__ int operator()(int x) const { return x; }
};

__global__ void __launch_bounds__(256, 3) k_fft_x_green(float2* __restrict__ grid, const float4* __restrict__ gridk,
                                                    int Nx, int Ny, int Nz, int B, int nzc, FFTPlan pl,
                                                    const float2* __restrict__ tw_global) {
    extern __shared__ float2 smem[];
    __shared__ int ly[64], lz[64], lmir[64];
    __shared__ int s_nl, s_np;  // lines, primary lines (whose points start the pairs)
    const int n = Nx;
    float2* tw = smem;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_global[i];
    const size_t G = (size_t)Nx * Ny * Nz;
    if (threadIdx.x == 0) {
        const int2 c = x_green_lines(blockIdx.x, Ny, Nz, B, nzc, ly, lz, lmir);
        s_nl = c.x;
        s_np = c.y;
    }
    __syncthreads();
    const int nl = s_nl, np = s_np;
    const int L6 = 6 * nl;  // lines in shared memory: grid-major
    float2* a = smem + n;
    float2* b = a + (size_t)L6 * n;
    for (int i = threadIdx.x; i < L6 * n; i += blockDim.x) {
        const int x = i / L6, q = i - x * L6;  // consecutive threads: consecutive lines (z runs)
        const int g = q / nl, l = q - g * nl;
        a[(size_t)q * n + x] = grid[(size_t)g * G + ((size_t)x * Ny + ly[l]) * Nz + lz[l]];
    }
    __syncthreads();
    float2* res = fft_lines(a, b, L6, pl, tw, false);
    x_green_pairs(res, nl, np, n, IdentitySlot(), ly, lz, lmir, gridk, Nx, Ny, Nz);
    __syncthreads();
    float2* other = (res == a) ? b : a;
    float2* out = fft_lines(res, other, L6, pl, tw, true);
    for (int i = threadIdx.x; i < L6 * n; i += blockDim.x) {
        const int x = i / L6, q = i - x * L6;
        const int g = q / nl, l = q - g * nl;
        grid[(size_t)g * G + ((size_t)x * Ny + ly[l]) * Nz + lz[l]] = out[(size_t)q * n + x];
    }
}

// Length-N1*N2 transforms of nlines rows (row stride ls) in place: forward
// leaves coefficient k = k2 + N2 k1 at slot k1 + N1 k2; the inverse runs the
// adjoint stages in reverse order, from that order back to natural order.
template <int N1, int N2>
__device__ __forceinline__ void rows_fwd(float2* buf, int nlines, int ls, const float2* tw) {
    for (int t = threadIdx.x; t < nlines * N1; t += blockDim.x) {
        const int l = t % nlines, n1 = t / nlines;
        float2* L = buf + l * ls + n1;
        float2 y[N2];
#pragma unroll
        for (int q = 0; q < N2; ++q) y[q] = L[q * N1];
        small_dft<N2>(y, false);
#pragma unroll
        for (int q = 0; q < N2; ++q) L[q * N1] = q == 0 ? y[0] : cmul(y[q], tw[n1 * q]);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nlines * N2; t += blockDim.x) {
        const int l = t % nlines, k2 = t / nlines;
        float2* L = buf + l * ls + k2 * N1;
        float2 y[N1];
#pragma unroll
        for (int q = 0; q < N1; ++q) y[q] = L[q];
        small_dft<N1>(y, false);
#pragma unroll
        for (int q = 0; q < N1; ++q) L[q] = y[q];
    }
    __syncthreads();
}

template <int N1, int N2>
__device__ __forceinline__ void rows_inv(float2* buf, int nlines, int ls, const float2* tw) {
    for (int t = threadIdx.x; t < nlines * N2; t += blockDim.x) {
        const int l = t % nlines, k2 = t / nlines;
        float2* L = buf + l * ls + k2 * N1;
        float2 y[N1];
#pragma unroll
        for (int q = 0; q < N1; ++q) y[q] = L[q];
        small_dft<N1>(y, true);
#pragma unroll
        for (int q = 0; q < N1; ++q) L[q] = y[q];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nlines * N1; t += blockDim.x) {
        const int l = t % nlines, n1 = t / nlines;
        float2* L = buf + l * ls + n1;
        float2 y[N2];
#pragma unroll
        for (int q = 0; q < N2; ++q) y[q] = q == 0 ? L[0] : cmul(L[q * N1], conjf2(tw[n1 * q]));
        small_dft<N2>(y, true);
#pragma unroll
        for (int q = 0; q < N2; ++q) L[q * N1] = y[q];
    }
    __syncthreads();
}

template <int N1, int N2>
struct DigitSlot {
    __device__ int operator()(int x) const { return x / N2 + N1 * (x % N2); }
};

// The fused x-pass for Nx = N1 * N2: one shared buffer, rows padded to N + 1.
template <int N1, int N2>
__global__ void __launch_bounds__(256, 3) k_fft_x_green_t(float2* __restrict__ grid, const float4* __restrict__ gridk,
                                                          int Ny, int Nz, int B, int nzc,
                                                          const float2* __restrict__ tw_global) {
    constexpr int n = N1 * N2, LS = n + 1;
    extern __shared__ float2 smem[];
    __shared__ int ly[64], lz[64], lmir[64];
    __shared__ int s_nl, s_np;
    float2* tw = smem;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_global[i];
    const size_t G = (size_t)n * Ny * Nz;
    if (threadIdx.x == 0) {
        const int2 c = x_green_lines(blockIdx.x, Ny, Nz, B, nzc, ly, lz, lmir);
        s_nl = c.x;
        s_np = c.y;
    }
    __syncthreads();
    const int nl = s_nl, np = s_np;
    const int L6 = 6 * nl;
    float2* a = smem + n;
    for (int i = threadIdx.x; i < L6 * n; i += blockDim.x) {
        const int x = i / L6, q = i - x * L6;
        const int g = q / nl, l = q - g * nl;
        a[(size_t)q * LS + x] = grid[(size_t)g * G + ((size_t)x * Ny + ly[l]) * Nz + lz[l]];
    }
    __syncthreads();
    rows_fwd<N1, N2>(a, L6, LS, tw);
    x_green_pairs(a, nl, np, LS, DigitSlot<N1, N2>(), ly, lz, lmir, gridk, n, Ny, Nz);
    __syncthreads();
    rows_inv<N1, N2>(a, L6, LS, tw);
    for (int i = threadIdx.x; i < L6 * n; i += blockDim.x) {
        const int x = i / L6, q = i - x * L6;
        const int g = q / nl, l = q - g * nl;
        grid[(size_t)g * G + ((size_t)x * Ny + ly[l]) * Nz + lz[l]] = a[(size_t)q * LS + x];
    }
}

// Launch of the fused x-pass: z-runs of B (4 unless tuned), fewer when the
// lines would not fit in shared memory.
static void fft_x_green(fsd_handle* h) {
    const int Nx = h->g.Nx, Ny = h->g.Ny, Nz = h->g.Nz;
    const FFTPlan px = make_fft_plan(Nx);
    const size_t cap = 200 * 1024;
    int B = (h->tune.set && h->tune.Bg > 0) ? h->tune.Bg : 4;
    while (B > 1 && sizeof(float2) * ((size_t)Nx + 2 * 12 * (size_t)B * Nx) > cap) --B;
    const int h2 = (Nz + 1) / 2;
    const int nzc = (h2 - 1 + B - 1) / B;
    const int nplanes = (Nz % 2 == 0) ? 2 : 1;
    const int nblocks = Ny * nzc + nplanes * (Ny / 2 + 1);
    const size_t shm = sizeof(float2) * ((size_t)Nx + 2 * 12 * (size_t)B * Nx);
    // Specialised line lengths keep one padded buffer (rows of Nx + 1).
    const size_t shm_t = sizeof(float2) * ((size_t)Nx + 12 * (size_t)B * (Nx + 1));
    auto go = [&](auto kern) {
        if (!smem_limit_ok((const void*)kern, shm_t, "k_fft_x_green_t shared memory")) return;
        count_launch();
        kern<<<nblocks, 256, shm_t, h->stream>>>(h->w.grid, h->w.gridk, Ny, Nz, B, nzc, h->w.twiddle);
    };
    switch (Nx) {
        case 72: go(k_fft_x_green_t<8, 9>); return;
        case 36: go(k_fft_x_green_t<4, 9>); return;
        case 27: go(k_fft_x_green_t<3, 9>); return;
        default: break;
    }
    if (!smem_limit_ok((const void*)k_fft_x_green, shm, "k_fft_x_green shared memory")) return;
    count_launch();
    k_fft_x_green<<<nblocks, 256, shm, h->stream>>>(h->w.grid, h->w.gridk, Nx, Ny, Nz, B, nzc, px, h->w.twiddle);
}

// ------------------------------------------------------ particle preparation
// Split the generalized force and map torque + stresslet to the couplet
// (Saddle_SplitGeneralizedF_kernel, Helper_Saddle.cu:108; Mobility_TS2C_kernel,
// Helper_Mobility.cu:294-336, including its torque sign flip).
__global__ void k_prep(const float* __restrict__ genF, int N, float4* f4, float4* c4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float* a = genF + 6 * i;
    const float* s = genF + 6 * N + 5 * i;
    f4[i] = make_float4(a[0], a[1], a[2], 0.0f);
    const float Lx = -a[3], Ly = -a[4], Lz = -a[5];
    const float Sxx = s[0], Sxy = s[1], Sxz = s[2], Syz = s[3], Syy = s[4];
    c4[2 * i] = make_float4(Sxx, Sxy + 0.5f * Lz, Sxz - 0.5f * Ly, Syz + 0.5f * Lx);
    c4[2 * i + 1] = make_float4(Syy, Sxy - 0.5f * Lz, Sxz + 0.5f * Ly, Syz - 0.5f * Lx);
}

// Stencil origin of each particle: the reference's first node
// x + 0 - P/2 + 1 - (P%2)(frac < 0.5) (Mobility.cu:242-248), wrapped.
__device__ __forceinline__ int3 stencil_origin(float4 p, const Box& b, int Nx, int Ny, int Nz, int P, float3* fr) {
    float3 f = make_fraction(make_float3(p.x, p.y, p.z), b);
    f.x *= (float)Nx;
    f.y *= (float)Ny;
    f.z *= (float)Nz;
    const int x = (int)f.x, y = (int)f.y, z = (int)f.z;
    const int Pd2 = P / 2;
    int sx = x - Pd2 + 1 - (P % 2) * ((f.x - (float)x) < 0.5f);
    int sy = y - Pd2 + 1 - (P % 2) * ((f.y - (float)y) < 0.5f);
    int sz = z - Pd2 + 1 - (P % 2) * ((f.z - (float)z) < 0.5f);
    if (fr) *fr = f;
    sx = ((sx % Nx) + Nx) % Nx;
    sy = ((sy % Ny) + Ny) % Ny;
    sz = ((sz % Nz) + Nz) % Nz;
    return make_int3(sx, sy, sz);
}

__global__ void k_origin_key(const float4* __restrict__ pos, int N, Box b, int Nx, int Ny, int Nz, int P, unsigned* key,
                             int* origin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int3 s = stencil_origin(pos[i], b, Nx, Ny, Nz, P, nullptr);
    key[i] = (unsigned)((s.x * Ny + s.y) * Nz + s.z);
    origin[3 * i] = s.x;
    origin[3 * i + 1] = s.y;
    origin[3 * i + 2] = s.z;
}

int mobility_bin_particles(fsd_handle* h, const float4* pos) {
    Workspace& w = h->w;
    const int N = h->p.N, Nx = h->g.Nx, Ny = h->g.Ny, Nz = h->g.Nz;
    count_launch();
    k_origin_key<<<(N + 255) / 256, 256, 0, h->stream>>>(pos, N, h->box, Nx, Ny, Nz, h->g.P, w.part_origin_key,
                                                        w.part_origin);
    counting_sort(w.part_origin_key, N, Nx * Ny * Nz, w.bin_count, w.bin_start, w.bin_fill, w.bin_parts,
                  w.scan_scratch, h->stream);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// --------------------------------------------------------------- spreading
struct SpreadArgs {
    const float4* pos;
    const float4* f4;
    const float4* c4;
    const unsigned* bin_start;
    const unsigned* bin_parts;
    const int* origin;
    float2* grid;
    Box box;
    int Nx, Ny, Nz, P;
    int TX, TY, TZ;
    float hx, hy, hz;
    float prefac, expfac;
    // Tile-relative separations: a staged particle keeps min_image(node(tile
    // origin) - p) and a node adds its fixed offset within the tile.  Valid
    // when the tile plus the stencil spans well under half the box on every
    // axis (so that sum is the minimum image itself); set by the host.
    bool local;
};

constexpr int kSpreadCap = 384;  // staged particles per pass

struct __align__(16) StagedParticle {  // read as four float4: (x, y, z, o), v[0:4], v[4:8], v[8:12]
    float x, y, z;
    int o;  // origin within the extended tile, packed (ox | oy << 10 | oz << 20)
    float v[12];
};

// Grid nodes of a tile gather from the particles staged in shared memory in
// cell order; cell_off[c] is the first staged index of extended cell c (the
// launch's dynamic shared memory, ncell + 1 entries).  The particles that
// reach a node are those whose stencil origin lies in the P^3 cells below
// it.  Two ways of visiting them, both adding each node's contributions in
// staged order (so both give the same sums):
//  ROWS = true   one node per thread; for each of its P x P (x, y) rows a
//                contiguous range of P cells, so a node visits exactly its
//                contributors (lanes diverge on uneven row lengths);
//  ROWS = false  a warp owns a 2 x 4 x 4 block of nodes; it ballots which
//                staged particles reach the block and takes them one at a
//                time, every lane reading the same particle (a shared-memory
//                broadcast) and adding it when its node lies in the stencil.
//                Needs TX % 2 == 0, TY % 4 == 0, TZ % 4 == 0.
template <bool ROWS>
__global__ void __launch_bounds__(256, ROWS ? 3 : 4) k_spread(SpreadArgs a) {
    __shared__ StagedParticle sp[kSpreadCap];
    __shared__ int so[ROWS ? 1 : kSpreadCap];  // packed origins, contiguous for the ballot
    __shared__ unsigned scan_sh[32];
    __shared__ unsigned s_total;
    extern __shared__ unsigned cell_off[];
    const int P = a.P;
    const int ntx = (a.Nx + a.TX - 1) / a.TX, nty = (a.Ny + a.TY - 1) / a.TY;
    int bid = blockIdx.x;
    const int tx = bid % ntx;
    bid /= ntx;
    const int ty = bid % nty;
    const int tz = bid / nty;
    const int x0 = tx * a.TX, y0 = ty * a.TY, z0 = tz * a.TZ;
    const float Ld2x0 = a.box.Lx / 2.0f, Ld2y0 = a.box.Ly / 2.0f, Ld2z0 = a.box.Lz / 2.0f;
    float3 pg0;  // position of the tile's origin node
    pg0.x = a.hx * x0 - Ld2x0;
    pg0.y = a.hy * y0 - Ld2y0;
    pg0.z = a.hz * z0 - Ld2z0;
    pg0.x = pg0.x + a.box.xy * pg0.y;
    const int EX = a.TX + P - 1, EY = a.TY + P - 1, EZ = a.TZ + P - 1;
    const int ex0 = x0 - (P - 1), ey0 = y0 - (P - 1), ez0 = z0 - (P - 1);
    const int ncell = EX * EY * EZ;
    const int nth = blockDim.x;
    const int cpt = (ncell + nth - 1) / nth;  // extended cells per thread, contiguous
    // Count staged particles per thread (deterministic order: cell order, then bin order).
    // The extended cells are walked with running coordinates (one division per
    // thread); ex0 + cx lies in [-(P - 1), 2 Nx) because TX <= Nx - P + 1, so
    // one conditional add or subtract wraps it.  Each cell's bin goes to
    // cell_bin for the staging pass.
    unsigned* cell_bin = cell_off + ncell + 1;
    unsigned mycount = 0;
    const int c_begin = threadIdx.x * cpt, c_end = min(ncell, (threadIdx.x + 1) * cpt);
    {
        int cz = c_begin % EZ, cy = (c_begin / EZ) % EY, cx = c_begin / (EZ * EY);
        for (int c = c_begin; c < c_end; ++c) {
            int gx = ex0 + cx, gy = ey0 + cy, gz = ez0 + cz;
            gx += gx < 0 ? a.Nx : (gx >= a.Nx ? -a.Nx : 0);
            gy += gy < 0 ? a.Ny : (gy >= a.Ny ? -a.Ny : 0);
            gz += gz < 0 ? a.Nz : (gz >= a.Nz ? -a.Nz : 0);
            const unsigned bin = (unsigned)((gx * a.Ny + gy) * a.Nz + gz);
            cell_bin[c] = bin;
            cell_off[c] = mycount;  // offset within this thread's cells; the block offset is added below
            mycount += a.bin_start[bin + 1] - a.bin_start[bin];
            if (++cz == EZ) {
                cz = 0;
                if (++cy == EY) {
                    cy = 0;
                    ++cx;
                }
            }
        }
    }
    // Block exclusive scan of counts.
    unsigned x = mycount;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scan_sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned s = (lane < (nth >> 5)) ? scan_sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        scan_sh[lane] = s;
        if (lane == 31) s_total = s;
    }
    __syncthreads();
    const unsigned myoff = (wid ? scan_sh[wid - 1] : 0u) + x - mycount;
    const unsigned total = s_total;
    for (int c = c_begin; c < c_end; ++c) cell_off[c] += myoff;
    if (threadIdx.x == 0) cell_off[ncell] = total;

    // This thread's node.
    int lx, ly, lz;
    int bx = 0, by = 0, bz = 0;  // the warp's node block (ROWS = false)
    if (ROWS) {
        lz = threadIdx.x % a.TZ;
        ly = (threadIdx.x / a.TZ) % a.TY;
        lx = threadIdx.x / (a.TZ * a.TY);
    } else {
        const int WZ = a.TZ >> 2, WY = a.TY >> 2;
        bz = 4 * (wid % WZ);
        by = 4 * ((wid / WZ) % WY);
        bx = 2 * (wid / (WZ * WY));
        lz = bz + (lane & 3);
        ly = by + ((lane >> 2) & 3);
        lx = bx + (lane >> 4);
    }
    const int nx = x0 + lx, ny = y0 + ly, nz = z0 + lz;
    const bool active = (lx < a.TX) && nx < a.Nx && ny < a.Ny && nz < a.Nz;
    const float Ld2x = a.box.Lx / 2.0f, Ld2y = a.box.Ly / 2.0f, Ld2z = a.box.Lz / 2.0f;
    float3 pg;
    pg.x = a.hx * nx - Ld2x;
    pg.y = a.hy * ny - Ld2y;
    pg.z = a.hz * nz - Ld2z;
    pg.x = pg.x + a.box.xy * pg.y;
    // offset of this node from the tile origin (the grid is sheared with the box)
    const float3 dn = make_float3(a.hx * lx + a.box.xy * (a.hy * ly), a.hy * ly, a.hz * lz);
    float acc[11];
#pragma unroll
    for (int c = 0; c < 11; ++c) acc[c] = 0.0f;

    for (unsigned chunk = 0; chunk < total; chunk += kSpreadCap) {
        // Stage this thread's particles that fall in [chunk, chunk + cap).
        unsigned k = myoff;
        int cz = c_begin % EZ, cy = (c_begin / EZ) % EY, cx = c_begin / (EZ * EY);
        for (int c = c_begin; c < c_end; ++c) {
            const unsigned bin = cell_bin[c];
            const unsigned q1 = a.bin_start[bin + 1];
            for (unsigned q = a.bin_start[bin]; q < q1; ++q, ++k) {
                if (k < chunk || k >= chunk + kSpreadCap) continue;
                const unsigned p = a.bin_parts[q];
                StagedParticle& s = sp[k - chunk];
                const float4 ps = a.pos[p];
                if (a.local) {
                    const float3 d = min_image(make_float3(pg0.x - ps.x, pg0.y - ps.y, pg0.z - ps.z), a.box);
                    s.x = d.x;
                    s.y = d.y;
                    s.z = d.z;
                } else {
                    s.x = ps.x;
                    s.y = ps.y;
                    s.z = ps.z;
                }
                s.o = cx | (cy << 10) | (cz << 20);
                if (!ROWS) so[k - chunk] = s.o;
                const float4 f = a.f4[p], c0 = a.c4[2 * p], c1 = a.c4[2 * p + 1];
                // pairs: (Fx,Fy) (Cxx,Cxy) (Cxz,Cyx) (Cyy,Cyz) (Czx,Czy) (Fz,0)
                s.v[0] = f.x; s.v[1] = f.y; s.v[2] = c0.x; s.v[3] = c0.y; s.v[4] = c0.z; s.v[5] = c1.y;
                s.v[6] = c1.x; s.v[7] = c0.w; s.v[8] = c1.z; s.v[9] = c1.w; s.v[10] = f.z; s.v[11] = 0.0f;
            }
            if (++cz == EZ) {
                cz = 0;
                if (++cy == EY) {
                    cy = 0;
                    ++cx;
                }
            }
        }
        __syncthreads();
        const unsigned cend = chunk + min((unsigned)kSpreadCap, total - chunk);
        if (!ROWS) {
            // Lane (i, j, k) of the warp holds node (bx + i, by + j, bz + k),
            // lane = 16 i + 4 j + k.  For the particle it examines, each lane
            // builds the mask of the warp's lanes inside that particle's
            // stencil (i in [dx - P + 1, dx], dx = cx - bx, and so on); the
            // warp then takes the particles whose mask is not empty in staged
            // order and reads the mask from the examining lane.
            const unsigned cnt = cend - chunk;
            const unsigned live = __ballot_sync(0xffffffffu, active);
            for (unsigned base = 0; base < cnt; base += 32) {
                unsigned lm = 0;
                if (base + lane < cnt) {
                    const int o = so[base + lane];
                    const int dx = (o & 1023) - bx, dy = ((o >> 10) & 1023) - by, dz = (o >> 20) - bz;
                    // bits [max(0, d - P + 1), min(w - 1, d)] of a w-bit row
                    auto span = [P](int d, int w) -> unsigned {
                        const int lo = max(0, d - P + 1), hi = min(w - 1, d);
                        return lo <= hi ? ((2u << hi) - (1u << lo)) : 0u;
                    };
                    const unsigned mx = span(dx, 2), my = span(dy, 4), mz = span(dz, 4);
                    const unsigned yz = mz * ((my & 1u) | ((my & 2u) << 3) | ((my & 4u) << 6) | ((my & 8u) << 9));
                    lm = yz * ((mx & 1u) | ((mx & 2u) << 15)) & live;
                }
                unsigned m = __ballot_sync(0xffffffffu, lm != 0);
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    const unsigned mask = __shfl_sync(0xffffffffu, lm, b);
                    if ((mask >> lane) & 1u) {
                        const float4* s4 = reinterpret_cast<const float4*>(&sp[base + b]);
                        const float4 sx = s4[0], v0 = s4[1], v1 = s4[2], v2 = s4[3];
                        const float3 r = a.local ? make_float3(sx.x + dn.x, sx.y + dn.y, sx.z + dn.z)
                                                 : min_image(make_float3(pg.x - sx.x, pg.y - sx.y, pg.z - sx.z), a.box);
                        const float rsq = r.x * r.x + r.y * r.y + r.z * r.z;
                        const float wgt = a.prefac * expf(-a.expfac * rsq);
                        acc[0] += wgt * v0.x;
                        acc[1] += wgt * v0.y;
                        acc[2] += wgt * v0.z;
                        acc[3] += wgt * v0.w;
                        acc[4] += wgt * v1.x;
                        acc[5] += wgt * v1.y;
                        acc[6] += wgt * v1.z;
                        acc[7] += wgt * v1.w;
                        acc[8] += wgt * v2.x;
                        acc[9] += wgt * v2.y;
                        acc[10] += wgt * v2.z;
                    }
                }
            }
        } else if (active) {
            for (int ix = 0; ix < P; ++ix) {
                for (int iy = 0; iy < P; ++iy) {
                    const int c0 = ((lx + ix) * EY + (ly + iy)) * EZ + lz;
                    const unsigned q0 = max(cell_off[c0], chunk), q1 = min(cell_off[c0 + P], cend);
                    for (unsigned q = q0; q < q1; ++q) {
                        const float4* s4 = reinterpret_cast<const float4*>(&sp[q - chunk]);
                        const float4 sx = s4[0], v0 = s4[1], v1 = s4[2], v2 = s4[3];
                        const float3 r = a.local ? make_float3(sx.x + dn.x, sx.y + dn.y, sx.z + dn.z)
                                                 : min_image(make_float3(pg.x - sx.x, pg.y - sx.y, pg.z - sx.z), a.box);
                        const float rsq = r.x * r.x + r.y * r.y + r.z * r.z;
                        const float wgt = a.prefac * expf(-a.expfac * rsq);
                        acc[0] += wgt * v0.x;
                        acc[1] += wgt * v0.y;
                        acc[2] += wgt * v0.z;
                        acc[3] += wgt * v0.w;
                        acc[4] += wgt * v1.x;
                        acc[5] += wgt * v1.y;
                        acc[6] += wgt * v1.z;
                        acc[7] += wgt * v1.w;
                        acc[8] += wgt * v2.x;
                        acc[9] += wgt * v2.y;
                        acc[10] += wgt * v2.z;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (active) {
        const size_t G = (size_t)a.Nx * a.Ny * a.Nz;
        const size_t g = ((size_t)nx * a.Ny + ny) * a.Nz + nz;
        a.grid[g] = make_float2(acc[0], acc[1]);
        a.grid[G + g] = make_float2(acc[2], acc[3]);
        a.grid[2 * G + g] = make_float2(acc[4], acc[5]);
        a.grid[3 * G + g] = make_float2(acc[6], acc[7]);
        a.grid[4 * G + g] = make_float2(acc[8], acc[9]);
        a.grid[5 * G + g] = make_float2(acc[10], 0.0f);
    }
}

// ------------------------------------------------------------- contraction
// One warp per particle: interpolate velocity (3) and velocity gradient (8)
// from the P^3 stencil (Mobility_WaveSpace_ContractU / ContractD,
// Mobility.cu:503-841).  Output per particle, 11 floats: u then the velocity
// gradient in the reference's transposed storage
// {XX, YX, ZX, ZY, YY, XY, XZ, YZ}.
// Warps take particles in the cell-list order (a permutation of 0..N-1), so
// the warps of a block read overlapping stencils through L1.  KP > 0 fixes the
// stencil width at compile time (the node index arithmetic then divides by a
// constant); KP = 0 reads it at run time.  With `local` (the stencil spans
// well under half the box) each node's separation is the stencil origin's
// minimum image plus the node's fixed offset in the sheared grid.
template <int KP>
__global__ void __launch_bounds__(256) k_contract(const float4* __restrict__ pos, const unsigned* __restrict__ order,
                                                  const float2* __restrict__ grid, int N, Box b, int Nx, int Ny,
                                                  int Nz, int Prun, float hx, float hy, float hz, float prefac,
                                                  float expfac, bool local, float* __restrict__ out) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= N) return;
    const int P = KP > 0 ? KP : Prun;
    const int i = (int)order[w];
    const float4 p = pos[i];
    const int3 s = stencil_origin(p, b, Nx, Ny, Nz, P, nullptr);
    const size_t G = (size_t)Nx * Ny * Nz;
    const float Ld2x = b.Lx / 2.0f, Ld2y = b.Ly / 2.0f, Ld2z = b.Lz / 2.0f;
    float3 r0;  // stencil origin node minus the particle, minimum image
    {
        float3 pg;
        pg.x = hx * s.x - Ld2x;
        pg.y = hy * s.y - Ld2y;
        pg.z = hz * s.z - Ld2z;
        pg.x = pg.x + b.xy * pg.y;
        r0 = min_image(make_float3(pg.x - p.x, pg.y - p.y, pg.z - p.z), b);
    }
    float acc[11];
#pragma unroll
    for (int c = 0; c < 11; ++c) acc[c] = 0.0f;
    const int P3 = P * P * P;
    for (int t = lane; t < P3; t += 32) {
        const int tz = t % P, ty = (t / P) % P, tx = t / (P * P);
        int ix = s.x + tx, iy = s.y + ty, iz = s.z + tz;
        ix -= (ix >= Nx) ? Nx : 0;
        iy -= (iy >= Ny) ? Ny : 0;
        iz -= (iz >= Nz) ? Nz : 0;
        float3 r;
        if (local) {
            r = make_float3(r0.x + (hx * tx + b.xy * (hy * ty)), r0.y + hy * ty, r0.z + hz * tz);
        } else {
            float3 pg;
            pg.x = hx * ix - Ld2x;
            pg.y = hy * iy - Ld2y;
            pg.z = hz * iz - Ld2z;
            pg.x = pg.x + b.xy * pg.y;
            r = min_image(make_float3(pg.x - p.x, pg.y - p.y, pg.z - p.z), b);
        }
        const float rsq = r.x * r.x + r.y * r.y + r.z * r.z;
        const float wgt = prefac * expf(-expfac * rsq);
        const size_t g = ((size_t)ix * Ny + iy) * Nz + iz;
        const float2 q0 = __ldg(grid + g), q1 = __ldg(grid + G + g), q2 = __ldg(grid + 2 * G + g),
                     q3 = __ldg(grid + 3 * G + g), q4 = __ldg(grid + 4 * G + g), q5 = __ldg(grid + 5 * G + g);
        // q0=(Ux,Uy) q1=(XX,XY) q2=(XZ,YX) q3=(YY,YZ) q4=(ZX,ZY) q5=(Uz,-)
        acc[0] += wgt * q0.x;
        acc[1] += wgt * q0.y;
        acc[2] += wgt * q5.x;
        acc[3] += wgt * q1.x;  // XX
        acc[4] += wgt * q2.y;  // YX
        acc[5] += wgt * q4.x;  // ZX
        acc[6] += wgt * q4.y;  // ZY
        acc[7] += wgt * q3.x;  // YY
        acc[8] += wgt * q1.y;  // XY
        acc[9] += wgt * q2.x;  // XZ
        acc[10] += wgt * q3.y; // YZ
    }
#pragma unroll
    for (int c = 0; c < 11; ++c) acc[c] = group_sum<32>(acc[c]);
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < 11; ++c) out[11 * i + c] = acc[c];
    }
}

// ------------------------------------------- real space, self and combine
// Group of 8 lanes per particle: real-space Ewald pair sum with linear table
// interpolation (Mobility_RealSpace_kernel, Mobility.cu:1046-1226), the self
// term, the optional wave-space part, then velocity gradient -> (W, E)
// (Mobility_D2WE_kernel) and generalized packing
// (Saddle_MakeGeneralizedU_kernel).
struct RealArgs {
    const float4* pos;
    const unsigned* order;  // particles in cell order
    const float4* f4;
    const float4* c4;
    const float* uwave;     // may be null
    const unsigned* nneigh;
    const unsigned* nlist;
    int stride;
    const float4* table;
    float self_x, self_y;
    float ewald_cut, ewald_dr;
    int ewald_n;
    Box box;
    int N;
    bool real;
    const float* saddle_x;  // may be null: adds x[11N + 6i + c] to U_i
    float* genU;
};

constexpr int kRealGroup = 8;

__global__ void __launch_bounds__(128) k_real_combine(RealArgs a) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / kRealGroup;
    const int gl = threadIdx.x % kRealGroup;
    const int N = a.N;
    const bool valid = gid < N;
    const int i = (int)a.order[valid ? gid : N - 1];
    float u[3] = {0, 0, 0}, D[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (a.real) {
        const float4 pi = a.pos[i];
        const float mindistSq = a.ewald_dr * a.ewald_dr, maxdistSq = a.ewald_cut * a.ewald_cut;
        const unsigned nn = valid ? a.nneigh[i] : 0u;
        const unsigned* row = a.nlist + (size_t)i * a.stride;
        for (unsigned q = gl; q < nn; q += kRealGroup) {
            const unsigned j = row[q];
            const float4 pj = a.pos[j];
            const float3 r = min_image(make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z), a.box);
            const float distSqr = r.x * r.x + r.y * r.y + r.z * r.z;
            if (!(distSqr < maxdistSq && distSqr >= mindistSq)) continue;
            const float dist = sqrtf(distSqr);
            const float4 Fj = a.f4[j];
            const float4 C0 = a.c4[2 * j], C1 = a.c4[2 * j + 1];
            // Clamped so that a distance rounding up to the cutoff stays inside the table.
            const int r_ind = min(max(__float2int_rd(a.ewald_n * (dist - a.ewald_dr) / (a.ewald_cut - a.ewald_dr)), 0),
                                  a.ewald_n - 1);
            const float4 t1m = __ldg(a.table + 2 * r_ind), t2m = __ldg(a.table + 2 * r_ind + 1);
            const float4 t1p = __ldg(a.table + 2 * r_ind + 2), t2p = __ldg(a.table + 2 * r_ind + 3);
            const float fac = dist / a.ewald_dr - r_ind - 1.0f;
            const float f1 = t1m.x + (t1p.x - t1m.x) * fac;
            const float f2 = t1m.y + (t1p.y - t1m.y) * fac;
            const float g1 = -(t1m.z + (t1p.z - t1m.z) * fac);
            const float g2 = -(t1m.w + (t1p.w - t1m.w) * fac);
            const float h1 = t2m.x + (t2p.x - t2m.x) * fac;
            const float h2 = t2m.y + (t2p.y - t2m.y) * fac;
            const float h3 = t2m.z + (t2p.z - t2m.z) * fac;
            const float Rx = r.x / dist, Ry = r.y / dist, Rz = r.z / dist;
            const float rdotf = Rx * Fj.x + Ry * Fj.y + Rz * Fj.z;
            const float Czz = -(C0.x + C1.x);
            // C.r and r.C with C = [[XX XY XZ][YX YY YZ][ZX ZY ZZ]] = [[c0x c0y c0z][c1y c1x c0w][c1z c1w Czz]]
            const float Cr_x = C0.x * Rx + C0.y * Ry + C0.z * Rz;
            const float Cr_y = C1.y * Rx + C1.x * Ry + C0.w * Rz;
            const float Cr_z = C1.z * Rx + C1.w * Ry + Czz * Rz;
            const float rC_x = C0.x * Rx + C1.y * Ry + C1.z * Rz;
            const float rC_y = C0.y * Rx + C1.x * Ry + C1.w * Rz;
            const float rC_z = C0.z * Rx + C0.w * Ry + Czz * Rz;
            const float rCr = Rx * Cr_x + Ry * Cr_y + Rz * Cr_z;
            u[0] += f1 * Fj.x + (f2 - f1) * rdotf * Rx;
            u[1] += f1 * Fj.y + (f2 - f1) * rdotf * Ry;
            u[2] += f1 * Fj.z + (f2 - f1) * rdotf * Rz;
            u[0] += g1 * (Cr_x - rCr * Rx) + g2 * (rC_x - 4.f * rCr * Rx);
            u[1] += g1 * (Cr_y - rCr * Ry) + g2 * (rC_y - 4.f * rCr * Ry);
            u[2] += g1 * (Cr_z - rCr * Rz) + g2 * (rC_z - 4.f * rCr * Rz);
            // Velocity gradient from force (Mobility.cu:1177-1184).
            D[0] += -g1 * (Rx * Fj.x - rdotf * Rx * Rx) - g2 * (rdotf + Fj.x * Rx - 4.f * rdotf * Rx * Rx);
            D[1] += -g1 * (Rx * Fj.y - rdotf * Rx * Ry) - g2 * (Fj.x * Ry - 4.f * rdotf * Rx * Ry);
            D[2] += -g1 * (Rx * Fj.z - rdotf * Rx * Rz) - g2 * (Fj.x * Rz - 4.f * rdotf * Rx * Rz);
            D[3] += -g1 * (Ry * Fj.z - rdotf * Ry * Rz) - g2 * (Fj.y * Rz - 4.f * rdotf * Ry * Rz);
            D[4] += -g1 * (Ry * Fj.y - rdotf * Ry * Ry) - g2 * (rdotf + Fj.y * Ry - 4.f * rdotf * Ry * Ry);
            D[5] += -g1 * (Ry * Fj.x - rdotf * Ry * Rx) - g2 * (Fj.y * Rx - 4.f * rdotf * Ry * Rx);
            D[6] += -g1 * (Rz * Fj.x - rdotf * Rz * Rx) - g2 * (Fj.z * Rx - 4.f * rdotf * Rz * Rx);
            D[7] += -g1 * (Rz * Fj.y - rdotf * Rz * Ry) - g2 * (Fj.z * Ry - 4.f * rdotf * Rz * Ry);
            // Velocity gradient from couplet (Mobility.cu:1186-1193).
            D[0] += h1 * (C0.x - 4.f * C0.x) + h2 * (Rx * Cr_x - rCr * Rx * Rx) +
                    h3 * (rCr + Cr_x * Rx + Rx * rC_x + rC_x * Rx - 6.f * rCr * Rx * Rx - C0.x);
            D[1] += h1 * (C0.y - 4.f * C1.y) + h2 * (Rx * Cr_y - rCr * Rx * Ry) +
                    h3 * (Cr_x * Ry + Rx * rC_y + rC_x * Ry - 6.f * rCr * Rx * Ry - C1.y);
            D[2] += h1 * (C0.z - 4.f * C1.z) + h2 * (Rx * Cr_z - rCr * Rx * Rz) +
                    h3 * (Cr_x * Rz + Rx * rC_z + rC_x * Rz - 6.f * rCr * Rx * Rz - C1.z);
            D[3] += h1 * (C0.w - 4.f * C1.w) + h2 * (Ry * Cr_z - rCr * Ry * Rz) +
                    h3 * (Cr_y * Rz + Ry * rC_z + rC_y * Rz - 6.f * rCr * Ry * Rz - C1.w);
            D[4] += h1 * (C1.x - 4.f * C1.x) + h2 * (Ry * Cr_y - rCr * Ry * Ry) +
                    h3 * (rCr + Cr_y * Ry + Ry * rC_y + rC_y * Ry - 6.f * rCr * Ry * Ry - C1.x);
            D[5] += h1 * (C1.y - 4.f * C0.y) + h2 * (Ry * Cr_x - rCr * Ry * Rx) +
                    h3 * (Cr_y * Rx + Ry * rC_x + rC_y * Rx - 6.f * rCr * Ry * Rx - C0.y);
            D[6] += h1 * (C1.z - 4.f * C0.z) + h2 * (Rz * Cr_x - rCr * Rz * Rx) +
                    h3 * (Cr_z * Rx + Rz * rC_x + rC_z * Rx - 6.f * rCr * Rz * Rx - C0.z);
            D[7] += h1 * (C1.w - 4.f * C0.w) + h2 * (Rz * Cr_y - rCr * Rz * Ry) +
                    h3 * (Cr_z * Ry + Rz * rC_y + rC_z * Ry - 6.f * rCr * Rz * Ry - C0.w);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) u[c] = group_sum<kRealGroup>(u[c]);
#pragma unroll
        for (int c = 0; c < 8; ++c) D[c] = group_sum<kRealGroup>(D[c]);
    }
    if (!valid || gl != 0) return;
    if (a.real) {
        const float4 F = a.f4[i], C0 = a.c4[2 * i], C1 = a.c4[2 * i + 1];
        u[0] += a.self_x * F.x;
        u[1] += a.self_x * F.y;
        u[2] += a.self_x * F.z;
        D[0] += a.self_y * (C0.x - 4.f * C0.x);
        D[1] += a.self_y * (C0.y - 4.f * C1.y);
        D[2] += a.self_y * (C0.z - 4.f * C1.z);
        D[3] += a.self_y * (C0.w - 4.f * C1.w);
        D[4] += a.self_y * (C1.x - 4.f * C1.x);
        D[5] += a.self_y * (C1.y - 4.f * C0.y);
        D[6] += a.self_y * (C1.z - 4.f * C0.z);
        D[7] += a.self_y * (C1.w - 4.f * C0.w);
    }
    if (a.uwave) {
        const float* w = a.uwave + 11 * i;
        u[0] = w[0] + u[0];
        u[1] = w[1] + u[1];
        u[2] = w[2] + u[2];
#pragma unroll
        for (int c = 0; c < 8; ++c) D[c] = w[3 + c] + D[c];
    }
    // D2WE (Helper_Mobility.cu:235-283): D0 = (Exx, Exy+Wz, Exz-Wy, Eyz+Wx), D1 = (Eyy, Exy-Wz, Exz+Wy, Eyz-Wx).
    const float W0 = 0.5f * (D[3] - D[7]);
    const float W1 = 0.5f * (D[6] - D[2]);
    const float W2 = 0.5f * (D[1] - D[5]);
    const float E0 = D[0];
    const float E1 = 0.5f * (D[1] + D[5]);
    const float E2 = 0.5f * (D[2] + D[6]);
    const float E3 = 0.5f * (D[3] + D[7]);
    const float E4 = D[4];
    float* o = a.genU + 6 * i;
    float add[6] = {0, 0, 0, 0, 0, 0};
    if (a.saddle_x) {
        const float* xs = a.saddle_x + 11 * N + 6 * i;
#pragma unroll
        for (int c = 0; c < 6; ++c) add[c] = xs[c];
    }
    o[0] = u[0] + add[0];
    o[1] = u[1] + add[1];
    o[2] = u[2] + add[2];
    o[3] = W0 + add[3];
    o[4] = W1 + add[4];
    o[5] = W2 + add[5];
    float* e = a.genU + 6 * N + 5 * i;
    e[0] = 2 * E0 + E4;
    e[1] = 2 * E1;
    e[2] = 2 * E2;
    e[3] = 2 * E3;
    e[4] = 2 * E4 + E0;
}

// ------------------------------------------------------------------ drivers
static void spread(fsd_handle* h, const float4* pos) {
    const GridParams& g = h->g;
    SpreadArgs a;
    a.pos = pos;
    a.f4 = h->w.f4;
    a.c4 = h->w.c4;
    a.bin_start = h->w.bin_start;
    a.bin_parts = h->w.bin_parts;
    a.origin = h->w.part_origin;
    a.grid = h->w.grid;
    a.box = h->box;
    a.Nx = g.Nx;
    a.Ny = g.Ny;
    a.Nz = g.Nz;
    a.P = g.P;
    if (h->tune.set && h->tune.TX > 0) {
        a.TX = h->tune.TX;
        a.TY = h->tune.TY;
        a.TZ = h->tune.TZ;
    } else {
        a.TZ = std::min(8, g.Nz - g.P + 1);
        a.TY = std::min(8, g.Ny - g.P + 1);
        a.TX = std::min(4, g.Nx - g.P + 1);
    }
    a.hx = g.hx;
    a.hy = g.hy;
    a.hz = g.hz;
    const float xisq = h->p.xi * h->p.xi;
    a.prefac = (2.0 * xisq / kPiRef / g.eta) * sqrtf(2.0 * xisq / kPiRef / g.eta);
    a.expfac = 2.0 * xisq / g.eta;
    // Node-particle separations stay below (T + P) cells per axis, plus the
    // tilt's x shift; below half the box they are their own minimum image.
    const float tilt = 1.0f + fabsf(h->box.xy);
    a.local = (a.TX + g.P) * tilt < 0.5f * g.Nx && (a.TY + g.P) * tilt < 0.5f * g.Ny &&
              (a.TZ + g.P) * tilt < 0.5f * g.Nz;
    const int ntiles = ((g.Nx + a.TX - 1) / a.TX) * ((g.Ny + a.TY - 1) / a.TY) * ((g.Nz + a.TZ - 1) / a.TZ);
    const size_t cell_bytes = sizeof(unsigned) * (2 * (size_t)(a.TX + g.P - 1) * (a.TY + g.P - 1) * (a.TZ + g.P - 1) + 1);
    const bool blocks = a.TX % 2 == 0 && a.TY % 4 == 0 && a.TZ % 4 == 0 && a.TX * a.TY * a.TZ == 256;
    count_launch();
    if (blocks && !(h->tune.set && h->tune.spread_rows))
        k_spread<false><<<ntiles, a.TX * a.TY * a.TZ, cell_bytes, h->stream>>>(a);
    else
        k_spread<true><<<ntiles, a.TX * a.TY * a.TZ, cell_bytes, h->stream>>>(a);
}

static void contract(fsd_handle* h, const float4* pos) {
    const GridParams& g = h->g;
    const float xisq = h->p.xi * h->p.xi;
    const float prefac = (2.0 * xisq / kPiRef / g.eta) * sqrtf(2.0 * xisq / kPiRef / g.eta);
    const float expfac = 2.0 * xisq / g.eta;
    const float quadW = g.hx * g.hy * g.hz;
    const int N = h->p.N;
    // node separations from the stencil origin reach (P - 1) cells per axis
    // plus the tilt's x shift; below half the box they are their own minimum image
    const float tilt = 1.0f + fabsf(h->box.xy);
    const bool local = (g.P + 1) * tilt < 0.5f * g.Nx && (g.P + 1) * tilt < 0.5f * g.Ny &&
                       (g.P + 1) * tilt < 0.5f * g.Nz;
    const unsigned grid = (unsigned)(((size_t)N * 32 + 255) / 256);
    count_launch();
    if (g.P == 6)
        k_contract<6><<<grid, 256, 0, h->stream>>>(pos, h->w.order, h->w.grid, N, h->box, g.Nx, g.Ny, g.Nz, g.P, g.hx,
                                                   g.hy, g.hz, quadW * prefac, expfac, local, h->w.uwave);
    else
        k_contract<0><<<grid, 256, 0, h->stream>>>(pos, h->w.order, h->w.grid, N, h->box, g.Nx, g.Ny, g.Nz, g.P, g.hx,
                                                   g.hy, g.hz, quadW * prefac, expfac, local, h->w.uwave);
}

void mobility_wave_from_spectrum(fsd_handle* h, const float4* pos) {
    {
        ProfRegion pr(h, R_FFT);
        fft3d(h, true, 6);
    }
    ProfRegion pr(h, R_CONTRACT);
    contract(h, pos);
}

void mobility_combine(fsd_handle* h, const float4* pos, const float* genF, float* genU, bool wave, bool real,
                      const float* saddle_x) {
    (void)genF;
    RealArgs r;
    r.pos = pos;
    r.order = h->w.order;
    r.f4 = h->w.f4;
    r.c4 = h->w.c4;
    r.uwave = wave ? h->w.uwave : nullptr;
    r.nneigh = h->w.nneigh;
    r.nlist = h->w.nlist;
    r.stride = h->w.nl_stride;
    r.table = h->d_ewald;
    r.self_x = h->self_x;
    r.self_y = h->self_y;
    r.ewald_cut = h->ewald_cut;
    r.ewald_dr = h->ewald_dr;
    r.ewald_n = h->ewald_n;
    r.box = h->box;
    r.N = h->p.N;
    r.real = real;
    r.saddle_x = saddle_x;
    r.genU = genU;
    const int N = h->p.N;
    count_launch();
    k_real_combine<<<(N * kRealGroup + 127) / 128, 128, 0, h->stream>>>(r);
}

// ---------------------------------------------------------------- autotuner
// On the first wave-space application with autotune set: time each candidate
// spreading tile and FFT line batch with CUDA events on the live grid (one
// warm-up, then the best of three) and keep the fastest.  Choices are cached
// per process for the grid shape and particle count, so all handles of a
// process agree.  The grid contents are overwritten; the caller spreads anew.
namespace {
std::mutex g_tune_mu;
std::map<std::array<int, 5>, TuneChoice> g_tune_cache;

float time_ms(fsd_handle* h, const std::function<void()>& f) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    f();
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a, h->stream);
        f();
        cudaEventRecord(b, h->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}
}  // namespace

static int autotune(fsd_handle* h, const float4* pos) {
    const GridParams& g = h->g;
    const std::array<int, 5> key{g.Nx, g.Ny, g.Nz, g.P, h->p.N};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            h->tune = it->second;
            return FSD_OK;
        }
    }
    TuneChoice best;
    best.set = true;
    float best_ms = 1e30f;
    const int tx_c[] = {1, 2, 4, 8}, ty_c[] = {2, 4, 8}, tz_c[] = {4, 8, 16, 32};
    for (int TX : tx_c)
        for (int TY : ty_c)
            for (int TZ : tz_c)
                for (int rows = 0; rows < 2; ++rows) {
                    const int T = TX * TY * TZ;
                    if (T < 64 || T > 256 || TX > g.Nx - g.P + 1 || TY > g.Ny - g.P + 1 || TZ > g.Nz - g.P + 1)
                        continue;
                    if (!rows && !(TX % 2 == 0 && TY % 4 == 0 && TZ % 4 == 0 && T == 256)) continue;
                    h->tune = TuneChoice{TX, TY, TZ, 0, 0, 0, rows, true};
                    const float ms = time_ms(h, [&] { spread(h, pos); });
                    if (ms < best_ms) {
                        best_ms = ms;
                        best.TX = TX;
                        best.TY = TY;
                        best.TZ = TZ;
                        best.spread_rows = rows;
                    }
                }
    std::vector<int> bxy, bz;
    for (int d = 8; d <= 32; ++d)
        if (g.Nz % d == 0) bxy.push_back(d);
    if (bxy.empty()) bxy.push_back(16);
    for (int d = 1; d * g.Nz <= 4096; ++d)
        if ((g.Nx * g.Ny) % d == 0 && sizeof(float2) * ((size_t)g.Nz + 2 * (size_t)d * g.Nz) <= 200 * 1024 &&
            d * g.Nz >= 256)
            bz.push_back(d);
    if (bz.empty()) bz.push_back(fft_batch_z(g.Nx, g.Ny, g.Nz));
    best_ms = 1e30f;
    for (int a : bxy)
        for (int b : bz) {
            h->tune = TuneChoice{best.TX, best.TY, best.TZ, a, b, 0, best.spread_rows, true};
            const float ms = time_ms(h, [&] {
                fft3d(h, false, 6);
                fft3d(h, true, 6);
            });
            if (ms < best_ms) {
                best_ms = ms;
                best.Bxy = a;
                best.Bz = b;
            }
        }
    best_ms = 1e30f;
    for (int bg : {1, 2, 4, 8}) {
        h->tune = best;
        h->tune.Bg = bg;
        const float ms = time_ms(h, [&] { fft_x_green(h); });
        if (ms < best_ms) {
            best_ms = ms;
            best.Bg = bg;
        }
    }
    h->tune = best;
    FSD_CHECK_CUDA(cudaGetLastError());
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache.emplace(key, best);
    return FSD_OK;
}

int mobility_apply(fsd_handle* h, const float4* pos, const float* genF, float* genU, int parts, const float* saddle_x,
                   bool rebin) {
    const int N = h->p.N;
    count_launch();
    k_prep<<<(N + 255) / 256, 256, 0, h->stream>>>(genF, N, h->w.f4, h->w.c4);
    const bool wave = parts & 1, real = parts & 2;
    if (wave) {
        {
            ProfRegion pr(h, R_SPREAD);
            if (rebin) {
                int st = mobility_bin_particles(h, pos);
                if (st != FSD_OK) return st;
            }
            if (h->p.autotune && !h->tune.set) {
                const int st = autotune(h, pos);
                if (st != FSD_OK) return st;
            }
            spread(h, pos);
        }
        {
            ProfRegion pr(h, R_FFT);
            fft3d(h, false, 6, true);  // z and y passes
        }
        {
            ProfRegion pr(h, R_GREEN);  // x pass, Green's function, inverse x pass
            fft_x_green(h);
        }
        {
            ProfRegion pr(h, R_FFT);
            fft3d(h, true, 6, true);  // y and z passes
        }
        {
            ProfRegion pr(h, R_CONTRACT);
            contract(h, pos);
        }
    }
    ProfRegion pr(h, R_REAL);
    mobility_combine(h, pos, genF, genU, wave, real, saddle_x);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

}  // namespace fsd
