// Internal declarations shared by the host and device translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fsd.h"

#define FSD_CHECK_CUDA(call)                                     \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) {                                 \
            fsd::set_last_cuda_error(e_, #call, __FILE__, __LINE__); \
            return FSD_ERR_CUDA;                                 \
        }                                                        \
    } while (0)

namespace fsd {

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);

// Kernel launches issued by this library (all handles, all threads).
void count_launch();
unsigned long long launch_count();

struct GridParams {
    int Nx = 0, Ny = 0, Nz = 0, P = 0;
    float ewald_cut = 0, gauss_m = 0, eta = 0, hx = 0, hy = 0, hz = 0;
};

int compute_grid_params(float xi, float error, float max_strain, float Lx, float Ly, float Lz, GridParams* g);
void ewald_table(float xi, float error, std::vector<float>& table, float* self_x, float* self_y, float* ewald_cut,
                 int* ewald_n, float* ewald_dr);
// Tabulated near-field resistance scalars: dist[1000], vals[1000*22].
const float* resistance_table_dist();
const float* resistance_table_vals();
constexpr int kResRows = 1000;
constexpr int kResFuncs = 22;
constexpr float kResMin = 0.000100f;   // Stokes_ResistanceTable.cc:37
constexpr float kResDr = 0.004305f;    // Stokes_ResistanceTable.cc:40

// Periodic box with an xy tilt, centred on the origin (HOOMD BoxDim semantics).
struct Box {
    float Lx, Ly, Lz, xy;
};

// Device-side bundle of what the pair kernels read.
struct PairList {
    const unsigned* nneigh;
    const unsigned* nlist;  // row-major, stride entries per particle
    int stride;
};

struct ResTable {
    const float* dist;
    const float* vals;
};

// Scratch owned by the handle, sized at creation.  Nothing is allocated per step.
struct Workspace {
    // neighbour list (row-major, nl_stride entries per particle)
    unsigned* nneigh = nullptr;
    unsigned* nlist = nullptr;
    int nl_stride = 0;
    int* nl_overflow = nullptr;    // device: largest count seen
    int* host_flag = nullptr;      // pinned host mirror of small flags
    unsigned* scan_scratch = nullptr;
    // cell list
    unsigned* part_cell = nullptr;
    unsigned* cell_count = nullptr;
    unsigned* cell_start = nullptr;
    unsigned* cell_fill = nullptr;
    unsigned* cell_parts = nullptr;
    size_t ncell_cap = 0;
    // particles in cell order (a permutation of 0..N-1, identity until the
    // first cell-list build): the order in which per-particle pair kernels
    // visit particles, so that neighbouring particles share the gathered data
    unsigned* order = nullptr;
    // the neighbour list restricted to r < rlub + nlist_buffer (same stride)
    unsigned* lub_n = nullptr;
    unsigned* lub_list = nullptr;
    // particles binned by spreading-stencil origin (one bin per grid node)
    unsigned* part_origin_key = nullptr;
    int* part_origin = nullptr;
    unsigned* bin_count = nullptr;
    unsigned* bin_start = nullptr;
    unsigned* bin_fill = nullptr;
    unsigned* bin_parts = nullptr;
    // wave space
    float2* grid = nullptr;        // 6 packed complex grids of G points
    float4* gridk = nullptr;       // wave vector and Green's scale per grid point
    float2* twiddle = nullptr;     // Nx + Ny + Nz twiddles
    // particle work arrays
    float4* f4 = nullptr;          // force per particle
    float4* c4 = nullptr;          // couplet, two float4 per particle
    float* uwave = nullptr;        // 11 per particle: wave-space u and velocity gradient
    // Krylov
    float* sx = nullptr;           // 17N work vectors
    float* sy = nullptr;
    float* sz = nullptr;
    float* V = nullptr;            // (restart + 1) x 17N basis
    float* Z = nullptr;            // restart x 17N preconditioned basis (flexible GMRES only)
    double* dred = nullptr;        // per-block partial sums
    double* hcol = nullptr;        // Hessenberg column, or the 2(j+1) dots of a delayed Gram-Schmidt pass
    unsigned* ticket = nullptr;    // last-block counter of the Gram-Schmidt update, zero between launches
    double* hcol2 = nullptr;       // re-orthogonalisation column
    void* gmres_state = nullptr;   // device GMRES state
    void* gmres_host = nullptr;    // pinned host mirror
    // preconditioner application
    float* pc_t = nullptr;         // 6N
    float* pc_y = nullptr;         // 6N
    // step-level vectors
    float* rhs = nullptr;          // 17N
    float* sol = nullptr;          // 17N (warm start carried between steps)
    float* rfd_rhs = nullptr;      // 17N
    float* rfd_sol = nullptr;      // 17N
    float* psi = nullptr;          // 6N random vector for the drift
    float4* pos_prime = nullptr;   // displaced positions for the drift
    float* vel = nullptr;          // 11N velocity scratch
    float* force = nullptr;        // 6N applied force scratch
    // Brownian
    float* lanczos_V = nullptr;    // (m_max + 1) x 11N
    float* lz_a = nullptr;         // 11N work vectors
    float* lz_b = nullptr;
    float* lz_c = nullptr;
    double* lz_dot = nullptr;      // device dot results
    double* lz_host = nullptr;     // pinned host copies
    // two-stage Runge-Kutta (integrator = 1 only)
    float4* rk_pos = nullptr;      // predictor positions, unwrapped
    float4* rk_posw = nullptr;     // predictor positions wrapped into the box (velocity evaluation)
    float* rk_ori = nullptr;       // predictor directors, 3N
    float* rk_vel = nullptr;       // velocity at the predictor, 11N
    float* rk_u1 = nullptr;        // velocity at the start of the step, 6N
    float* rk_noise = nullptr;     // angular noise of the step, 3N
};
// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device.  Function attributes are per device, so the record is kept
// per (kernel, device); limits at or below the 48 KiB default need no call.
inline cudaError_t ensure_smem_limit(const void* func, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> set;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = set[std::make_pair(func, dev)];
    if (cur >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// ensure_smem_limit for launch sites without a status return: a failure is
// recorded as the library's last CUDA error and the caller skips the launch
// (the enclosing entry point then reports FSD_ERR_CUDA through its
// cudaGetLastError check).
inline bool smem_limit_ok(const void* func, size_t bytes, const char* what) {
    const cudaError_t e = ensure_smem_limit(func, bytes);
    if (e == cudaSuccess) return true;
    set_last_cuda_error(e, what, __FILE__, __LINE__);
    return false;
}

}  // namespace fsd

// Launch shapes chosen by the autotuner (0 = built-in defaults).
struct TuneChoice {
    int TX = 0, TY = 0, TZ = 0;  // spreading tile
    int Bxy = 0, Bz = 0;         // FFT lines per block (x/y passes, z pass)
    int Bg = 0;                  // z-run length of the fused x-pass + Green kernel
    int spread_rows = 0;         // 1: one node per thread walking stencil rows; 0: warp node blocks
    bool set = false;
};

struct fsd_handle {
    fsd_params p;
    fsd::Box box;
    cudaStream_t stream = nullptr;
    int device = 0;                // CUDA device current at fsd_create
    fsd::GridParams g;
    float self_x = 0, self_y = 0, ewald_cut = 0, ewald_dr = 0;
    int ewald_n = 0;
    std::vector<float> ewald_host;
    float4* d_ewald = nullptr;
    float* d_res_dist = nullptr;
    float* d_res_vals = nullptr;
    fsd::Workspace w;
    fsd_solve_info info{};
    bool nlist_valid = false;
    bool pc_valid = false;
    uint32_t seed_hashed = 0;
    float ichol_relaxer = 1.0f;
    int m_lanczos_ff = 2, m_lanczos_nf = 2;
    void* ichol = nullptr;     // preconditioner state (precond.cu)
    void* learned = nullptr;   // block-sparse preconditioner state (learned.cu)
    TuneChoice tune;
    void* profiler = nullptr;  // region timers (profile.cpp)
};
