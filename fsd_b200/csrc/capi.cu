// C ABI entry points (include/fsd.h): handle lifecycle and the operator-level
// calls.  Time stepping lives in integrator.cu.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>

#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_learned.h"
#include "fsd_mpnn.h"
#include "fsd_solver.h"
#include "fsd_profile.h"

namespace fsd {

static thread_local char g_last_error[512] = "";
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    snprintf(g_last_error, sizeof(g_last_error), "%s (%s) at %s:%d: %s", cudaGetErrorName(e), what, file, line,
             cudaGetErrorString(e));
}

static int neighbor_stride_for(const fsd_params& p, float rlist) {
    const double V = (double)p.Lx * p.Ly * p.Lz;
    const double expected = 4.0 / 3.0 * M_PI * rlist * rlist * rlist * p.N / V;
    int s = (int)(1.6 * expected) + 48;
    s = (s + 31) / 32 * 32;
    return std::min(s, std::max(32, ((p.N + 31) / 32) * 32));
}

template <class T> static int dalloc(T** p, size_t n) {
    if (n == 0) n = 1;
    FSD_CHECK_CUDA(cudaMalloc((void**)p, sizeof(T) * n));
    return FSD_OK;
}

#define FSD_TRY(x)                  \
    do {                            \
        int s_ = (x);               \
        if (s_ != FSD_OK) return s_; \
    } while (0)

static int alloc_nlist(fsd_handle* h, int stride) {
    Workspace& w = h->w;
    if (w.nlist) cudaFree(w.nlist);
    if (w.lub_list) cudaFree(w.lub_list);
    w.nlist = nullptr;
    w.lub_list = nullptr;
    w.nl_stride = stride;
    FSD_TRY(dalloc(&w.nlist, (size_t)h->p.N * stride));
    return dalloc(&w.lub_list, (size_t)h->p.N * stride);
}

static int allocate(fsd_handle* h) {
    Workspace& w = h->w;
    const int N = h->p.N;
    const size_t G = (size_t)h->g.Nx * h->g.Ny * h->g.Nz;
    const float rlist = h->ewald_cut + h->p.nlist_buffer;
    FSD_TRY(dalloc(&w.nneigh, N));
    FSD_TRY(alloc_nlist(h, neighbor_stride_for(h->p, rlist)));
    FSD_TRY(dalloc(&w.nl_overflow, 1));
    FSD_CHECK_CUDA(cudaMallocHost(&w.host_flag, sizeof(int) * 4));
    // Cell capacity for the untilted box (tilting only removes cells).
    const int3 nc = cell_dims(Box{h->box.Lx, h->box.Ly, h->box.Lz, 0.0f}, rlist);
    w.ncell_cap = (nc.x >= 3 && nc.y >= 3 && nc.z >= 3) ? (size_t)nc.x * nc.y * nc.z : 0;
    const size_t nbins = std::max(w.ncell_cap, G);
    FSD_TRY(dalloc(&w.scan_scratch, scan_scratch_elems((int)nbins + 1)));
    FSD_TRY(dalloc(&w.part_cell, N));
    FSD_TRY(dalloc(&w.cell_count, w.ncell_cap + 1));
    FSD_TRY(dalloc(&w.cell_start, w.ncell_cap + 1));
    FSD_TRY(dalloc(&w.cell_fill, w.ncell_cap + 1));
    FSD_TRY(dalloc(&w.cell_parts, N));
    FSD_TRY(dalloc(&w.order, N));
    FSD_TRY(dalloc(&w.lub_n, N));
    FSD_TRY(init_particle_order(h));
    FSD_TRY(dalloc(&w.part_origin_key, N));
    FSD_TRY(dalloc(&w.part_origin, 3 * (size_t)N));
    FSD_TRY(dalloc(&w.bin_count, G + 1));
    FSD_TRY(dalloc(&w.bin_start, G + 1));
    FSD_TRY(dalloc(&w.bin_fill, G + 1));
    FSD_TRY(dalloc(&w.bin_parts, N));
    FSD_TRY(dalloc(&w.grid, 6 * G));
    FSD_TRY(dalloc(&w.gridk, G));
    FSD_TRY(dalloc(&w.twiddle, (size_t)h->g.Nx + h->g.Ny + h->g.Nz));
    FSD_TRY(dalloc(&w.f4, N));
    FSD_TRY(dalloc(&w.c4, 2 * (size_t)N));
    FSD_TRY(dalloc(&w.uwave, 11 * (size_t)N));
    const size_t n17 = 17 * (size_t)N;
    FSD_TRY(dalloc(&w.sx, n17));
    FSD_TRY(dalloc(&w.sy, n17));
    FSD_TRY(dalloc(&w.sz, n17));
    const int m = std::min(h->p.gmres_restart, kMaxRestart);
    FSD_TRY(dalloc(&w.V, (size_t)(m + 1) * krylov_ld(N)));
    if (h->p.precond == FSD_PRECOND_LEARNED && h->p.learned_inner > 0)  // flexible GMRES keeps M^-1 v_j
        FSD_TRY(dalloc(&w.Z, (size_t)m * krylov_ld(N)));
    FSD_TRY(dalloc(&w.dred, (size_t)2 * (kMaxRestart + 2) * 512));
    FSD_TRY(dalloc(&w.hcol, 2 * (kMaxRestart + 2)));
    FSD_TRY(dalloc(&w.ticket, 1));
    FSD_CHECK_CUDA(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned), h->stream));
    FSD_TRY(dalloc(&w.hcol2, kMaxRestart + 2));
    FSD_TRY(gmres_alloc(h));
    FSD_TRY(dalloc(&w.pc_t, 6 * (size_t)N));
    FSD_TRY(dalloc(&w.pc_y, 6 * (size_t)N));
    FSD_TRY(dalloc(&w.rhs, n17));
    FSD_TRY(dalloc(&w.sol, n17));
    FSD_TRY(dalloc(&w.rfd_rhs, n17));
    FSD_TRY(dalloc(&w.rfd_sol, n17));
    FSD_TRY(dalloc(&w.psi, 6 * (size_t)N));
    FSD_TRY(dalloc(&w.pos_prime, N));
    FSD_TRY(dalloc(&w.vel, 11 * (size_t)N));
    FSD_TRY(dalloc(&w.force, 6 * (size_t)N));
    FSD_TRY(dalloc(&w.lanczos_V, (size_t)(h->p.lanczos_max + 2) * 11 * N));
    FSD_TRY(dalloc(&w.lz_a, 11 * (size_t)N));
    FSD_TRY(dalloc(&w.lz_b, 11 * (size_t)N));
    FSD_TRY(dalloc(&w.lz_c, 11 * (size_t)N));
    FSD_TRY(dalloc(&w.lz_dot, 4096));
    FSD_CHECK_CUDA(cudaMallocHost(&w.lz_host, sizeof(double) * 4096));
    FSD_CHECK_CUDA(cudaMemsetAsync(w.sol, 0, sizeof(float) * n17, h->stream));
    if (h->p.integrator == 1) {
        FSD_TRY(dalloc(&w.rk_pos, N));
        FSD_TRY(dalloc(&w.rk_posw, N));
        FSD_TRY(dalloc(&w.rk_ori, 3 * (size_t)N));
        FSD_TRY(dalloc(&w.rk_vel, 11 * (size_t)N));
        FSD_TRY(dalloc(&w.rk_u1, 6 * (size_t)N));
        FSD_TRY(dalloc(&w.rk_noise, 3 * (size_t)N));
    }
    FSD_TRY(precond_alloc(h));
    return FSD_OK;
}

static void release(fsd_handle* h) {
    Workspace& w = h->w;
    void* dev[] = {w.nneigh, w.nlist, w.nl_overflow, w.scan_scratch, w.part_cell, w.cell_count, w.cell_start,
                   w.cell_fill, w.cell_parts, w.order, w.lub_n, w.lub_list, w.part_origin_key, w.part_origin, w.bin_count, w.bin_start, w.bin_fill,
                   w.bin_parts, w.grid, w.gridk, w.twiddle, w.f4, w.c4, w.uwave, w.sx, w.sy, w.sz, w.V, w.Z, w.dred,
                   w.hcol, w.hcol2, w.ticket, w.gmres_state, w.pc_t, w.pc_y, w.rhs, w.sol, w.rfd_rhs, w.rfd_sol, w.psi,
                   w.pos_prime, w.vel, w.force, w.lanczos_V, w.lz_a, w.lz_b, w.lz_c, w.lz_dot, h->d_ewald,
                   h->d_res_dist, h->d_res_vals, w.rk_pos, w.rk_posw, w.rk_ori, w.rk_vel, w.rk_u1, w.rk_noise};
    for (void* p : dev)
        if (p) cudaFree(p);
    if (w.host_flag) cudaFreeHost(w.host_flag);
    if (w.gmres_host) cudaFreeHost(w.gmres_host);
    if (w.lz_host) cudaFreeHost(w.lz_host);
    precond_free(h);
    learned_free(h);
    profile_destroy(h);
}

}  // namespace fsd

using namespace fsd;

extern "C" {

void fsd_default_params(fsd_params* p) {
    memset(p, 0, sizeof(*p));
    p->xi = 0.5f;
    p->error = 1e-3f;
    p->max_strain = 0.5f;
    p->solver_tol = 1e-3f;
    p->lanczos_tol = 1e-3f;
    p->rfd_epsilon = 1e-3f;
    p->T = 1.0f;
    p->dt = 1e-4f;
    p->seed = 0;
    p->ndsr = 1e-1f;
    p->kappa = 1.0f / 0.05f;
    p->k_n = 1e4f;
    p->beta_AF = 0.0f;
    p->epsq = 1e-5f;
    p->N_mix = 1;
    p->coef_B1_mask = 1.0f;
    p->coef_B2_mask = 1.0f;
    p->gmres_restart = 50;
    p->gmres_max_iter = 1000;
    p->lanczos_max = 100;
    p->precond = FSD_PRECOND_ICHOL;
    p->force_mode = FSD_FORCE_INTERPARTICLE;
    p->kgrid_pi_ref = 1;
    p->rlub = 4.0f;
    p->rp = 2.1f;
    p->nlist_buffer = 0.4f;
    p->ichol_local_shift = 1;
    p->ichol_gain_limit = 100.0f;
    p->learned_inner = 4;
    p->learned_poly = 0;
    p->poly_interval = 0.05f;
    p->friction_type = 0;
    p->friction_h0 = 0.0f;
    for (int k = 0; k < 6; ++k) p->friction_alpha[k] = 0.0f;
    p->integrator = 0;
}

// The resistance table with the TYPE1 friction patch (Stokes::setFriction,
// Stokes.cc:1132-1191): for every tabulated distance whose gap h = r - 2 is
// at most h0, alpha_k (2 h^2/h0^3 - 3 h/h0^2 + 1/h) is added in magnitude to
// YA11, YA12, YB11, YB12, YC11 and YC12 (entries 3, 4, 5, 6, 9, 10; the signs
// follow the tabulated functions' signs).  The bracket is evaluated in double
// from single-precision h and powers of h0, then rounded to single precision,
// as the reference's float/double mix does.
static void resistance_table_for(const fsd_params* p, std::vector<float>& dist, std::vector<float>& vals) {
    dist.assign(resistance_table_dist(), resistance_table_dist() + kResRows);
    vals.assign(resistance_table_vals(), resistance_table_vals() + (size_t)kResRows * kResFuncs);
    if (p->friction_type != 1) return;
    const float h0 = p->friction_h0;
    const float h02 = h0 * h0;
    const float h03 = h0 * h02;
    const int slot[6] = {3, 4, 5, 6, 9, 10};
    const float sign[6] = {1.f, -1.f, -1.f, 1.f, 1.f, 1.f};
    for (int i = 0; i < kResRows; ++i) {
        const float h = (float)((double)dist[i] - 2.0);
        if (!(h <= h0)) continue;
        const float h2 = h * h;
        const double bracket = 2.0 / h03 * h2 - 3.0 / h02 * h + 1.0 / h;
        for (int k = 0; k < 6; ++k) {
            const float add = (float)(p->friction_alpha[k] * bracket);
            float& v = vals[(size_t)kResFuncs * i + slot[k]];
            v = sign[k] > 0 ? v + add : v - add;
        }
    }
}

int fsd_resistance_table(const fsd_params* p, float* dist, float* vals) {
    if (!p || !dist || !vals || p->friction_type < 0 || p->friction_type > 1) return FSD_ERR_BAD_PARAMS;
    std::vector<float> d, v;
    resistance_table_for(p, d, v);
    std::copy(d.begin(), d.end(), dist);
    std::copy(v.begin(), v.end(), vals);
    return FSD_OK;
}

const char* fsd_status_string(int status) {
    switch (status) {
        case FSD_OK: return "ok";
        case FSD_ERR_BAD_PARAMS: return "bad parameters";
        case FSD_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA error";
        case FSD_ERR_GMRES_MAXIT: return "GMRES reached its iteration limit";
        case FSD_ERR_LANCZOS_MAXIT: return "Lanczos did not converge";
        case FSD_ERR_ICHOL: return "incomplete Cholesky failed";
        case FSD_ERR_NLIST_OVERFLOW: return "neighbour list overflow";
        case FSD_ERR_DEVICE_WAIT: return "device-side wait timed out";
        case FSD_ERR_ALLOC: return "allocation failed";
        case FSD_ERR_BREAKDOWN: return "Krylov breakdown or non-finite value";
        default: return "unknown status";
    }
}

int fsd_pse_setup(const fsd_params* p, fsd_pse_info* info, float* host_table, size_t n_floats) {
    if (!p || !info || !(p->xi > 0) || !(p->error > 0 && p->error < 1)) return FSD_ERR_BAD_PARAMS;
    GridParams g;
    const int st = compute_grid_params(p->xi, p->error, p->max_strain, p->Lx, p->Ly, p->Lz, &g);
    if (st != FSD_OK) return st;
    std::vector<float> tab;
    float sx, sy, cut, dr;
    int n;
    ewald_table(p->xi, p->error, tab, &sx, &sy, &cut, &n, &dr);
    info->Nx = g.Nx;
    info->Ny = g.Ny;
    info->Nz = g.Nz;
    info->P = g.P;
    info->ewald_cut = cut;
    info->gauss_m = g.gauss_m;
    info->eta = g.eta;
    info->hx = g.hx;
    info->hy = g.hy;
    info->hz = g.hz;
    info->self_x = sx;
    info->self_y = sy;
    info->ewald_n = n;
    info->ewald_dr = dr;
    if (host_table) {
        if (n_floats < tab.size()) return FSD_ERR_BAD_PARAMS;
        memcpy(host_table, tab.data(), sizeof(float) * tab.size());
    }
    return FSD_OK;
}

int fsd_rcm_order(int n, const int* rowptr, const int* col, int* perm) {
    if (n < 0 || (n > 0 && (!rowptr || !col || !perm))) return FSD_ERR_BAD_PARAMS;
    std::vector<int> rp(rowptr, rowptr + n + 1), cl(col, col + rowptr[n]), out;
    for (int v : cl)
        if (v < 0 || v >= n) return FSD_ERR_BAD_PARAMS;
    rcm_order(n, rp, cl, out);
    std::copy(out.begin(), out.end(), perm);
    return FSD_OK;
}

int fsd_create(const fsd_params* p, void* stream, fsd_handle** out) {
    if (!p || !out) return FSD_ERR_BAD_PARAMS;
    *out = nullptr;
    if (p->N < 1 || !(p->Lx > 0 && p->Ly > 0 && p->Lz > 0) || !(p->xi > 0) || !(p->error > 0 && p->error < 1))
        return FSD_ERR_BAD_PARAMS;
    if (p->gmres_restart < 1 || p->gmres_restart > kMaxRestart || p->lanczos_max < 4) return FSD_ERR_BAD_PARAMS;
    if (p->learned_inner < 0 || p->learned_inner > kMaxInner) return FSD_ERR_BAD_PARAMS;
    if (p->learned_poly < 0 || p->learned_poly == 1 || p->learned_poly > kMaxPoly) return FSD_ERR_BAD_PARAMS;
    if (!(p->poly_interval >= 0.f && p->poly_interval < 1.f)) return FSD_ERR_BAD_PARAMS;
    if (p->friction_type < 0 || p->friction_type > 1 || (p->friction_type == 1 && !(p->friction_h0 > 0.f)))
        return FSD_ERR_BAD_PARAMS;
    if (p->integrator < 0 || p->integrator > 1) return FSD_ERR_BAD_PARAMS;
    fsd_handle* h = new fsd_handle();
    h->p = *p;
    h->stream = (cudaStream_t)stream;
    cudaGetDevice(&h->device);
    h->box = Box{p->Lx, p->Ly, p->Lz, p->xy};
    int st = compute_grid_params(p->xi, p->error, p->max_strain, p->Lx, p->Ly, p->Lz, &h->g);
    if (st != FSD_OK) {
        delete h;
        return st;
    }
    ewald_table(p->xi, p->error, h->ewald_host, &h->self_x, &h->self_y, &h->ewald_cut, &h->ewald_n, &h->ewald_dr);
    // Seed hash of the Stokes constructor (Stokes.cc:74).
    uint32_t s = p->seed;
    s = s * 0x12345677u + 0x12345u;
    s ^= (s >> 16);
    s *= 0x45679u;
    h->seed_hashed = s;
    st = allocate(h);
    if (st == FSD_OK) {
        const size_t tb = h->ewald_host.size() * sizeof(float);
        if (cudaMalloc(&h->d_ewald, tb) != cudaSuccess || cudaMalloc(&h->d_res_dist, sizeof(float) * kResRows) ||
            cudaMalloc(&h->d_res_vals, sizeof(float) * kResRows * kResFuncs)) {
            st = FSD_ERR_ALLOC;
        } else {
            cudaMemcpyAsync(h->d_ewald, h->ewald_host.data(), tb, cudaMemcpyHostToDevice, h->stream);
            std::vector<float> tdist, tvals;
            resistance_table_for(p, tdist, tvals);
            cudaMemcpyAsync(h->d_res_dist, tdist.data(), sizeof(float) * kResRows, cudaMemcpyHostToDevice, h->stream);
            cudaMemcpyAsync(h->d_res_vals, tvals.data(), sizeof(float) * kResRows * kResFuncs, cudaMemcpyHostToDevice,
                            h->stream);
            fill_twiddles(h);
            mobility_set_gridk(h);
            if (cudaStreamSynchronize(h->stream) != cudaSuccess) st = FSD_ERR_CUDA;
        }
    }
    if (st != FSD_OK) {
        release(h);
        delete h;
        return st;
    }
    *out = h;
    return FSD_OK;
}

void fsd_destroy(fsd_handle* h) {
    if (!h) return;
    cudaStreamSynchronize(h->stream);
    release(h);
    delete h;
}

unsigned long long fsd_launch_count(void) { return launch_count(); }

int fsd_set_stream(fsd_handle* h, void* stream) {
    if (!h) return FSD_ERR_BAD_PARAMS;
    h->stream = (cudaStream_t)stream;
    return FSD_OK;
}

int fsd_set_box(fsd_handle* h, float Lx, float Ly, float Lz, float xy) {
    if (!h) return FSD_ERR_BAD_PARAMS;
    // The grid and Ewald parameters are fixed at creation (Stokes.cc:136);
    // only the tilt may change afterwards.
    if (Lx != h->p.Lx || Ly != h->p.Ly || Lz != h->p.Lz) return FSD_ERR_BAD_PARAMS;
    h->box.xy = xy;
    h->p.xy = xy;
    h->nlist_valid = false;
    mobility_set_gridk(h);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

int fsd_set_temperature(fsd_handle* h, float T) {
    if (!h || !(T >= 0)) return FSD_ERR_BAD_PARAMS;
    h->p.T = T;
    return FSD_OK;
}

int fsd_get_pse_info(const fsd_handle* h, fsd_pse_info* info) {
    if (!h || !info) return FSD_ERR_BAD_PARAMS;
    info->Nx = h->g.Nx;
    info->Ny = h->g.Ny;
    info->Nz = h->g.Nz;
    info->P = h->g.P;
    info->ewald_cut = h->ewald_cut;
    info->gauss_m = h->g.gauss_m;
    info->eta = h->g.eta;
    info->hx = h->g.hx;
    info->hy = h->g.hy;
    info->hz = h->g.hz;
    info->self_x = h->self_x;
    info->self_y = h->self_y;
    info->ewald_n = h->ewald_n;
    info->ewald_dr = h->ewald_dr;
    return FSD_OK;
}

int fsd_get_solve_info(const fsd_handle* h, fsd_solve_info* info) {
    if (!h || !info) return FSD_ERR_BAD_PARAMS;
    *info = h->info;
    const LearnedState* ls = (const LearnedState*)h->learned;
    info->poly_source = ls ? ls->poly_source : 0;
    info->poly_loss_net = ls ? ls->poly_loss_net : -1.f;
    info->poly_loss_fit = ls ? ls->poly_loss_fit : -1.f;
    info->poly_ratio = ls ? ls->poly_ratio : -1.f;
    return FSD_OK;
}

namespace {
struct CheckpointHeader {
    uint32_t magic;    // 'FSDC'
    uint32_t version;  // 1
    int32_t N;
    int32_t m_lanczos_ff, m_lanczos_nf;
    float ichol_relaxer;
};
constexpr uint32_t kCheckpointMagic = 0x43445346u;
}  // namespace

size_t fsd_checkpoint_size(const fsd_handle* h) {
    if (!h) return 0;
    return sizeof(CheckpointHeader) + sizeof(float) * 17 * (size_t)h->p.N;
}

int fsd_checkpoint_save(fsd_handle* h, void* host, size_t bytes) {
    if (!h || !host || bytes < fsd_checkpoint_size(h)) return FSD_ERR_BAD_PARAMS;
    CheckpointHeader hd{kCheckpointMagic, 1u, h->p.N, h->m_lanczos_ff, h->m_lanczos_nf, h->ichol_relaxer};
    std::memcpy(host, &hd, sizeof(hd));
    float* sol = reinterpret_cast<float*>(static_cast<char*>(host) + sizeof(hd));
    FSD_CHECK_CUDA(cudaMemcpyAsync(sol, h->w.sol, sizeof(float) * 17 * (size_t)h->p.N, cudaMemcpyDeviceToHost,
                                   h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return FSD_OK;
}

int fsd_checkpoint_load(fsd_handle* h, const void* host, size_t bytes) {
    if (!h || !host || bytes < fsd_checkpoint_size(h)) return FSD_ERR_BAD_PARAMS;
    CheckpointHeader hd;
    std::memcpy(&hd, host, sizeof(hd));
    if (hd.magic != kCheckpointMagic || hd.version != 1u || hd.N != h->p.N || hd.m_lanczos_ff < 1 ||
        hd.m_lanczos_nf < 1 || !(hd.ichol_relaxer > 0.f))
        return FSD_ERR_BAD_PARAMS;
    const float* sol = reinterpret_cast<const float*>(static_cast<const char*>(host) + sizeof(hd));
    FSD_CHECK_CUDA(cudaMemcpyAsync(h->w.sol, sol, sizeof(float) * 17 * (size_t)h->p.N, cudaMemcpyHostToDevice,
                                   h->stream));
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    h->m_lanczos_ff = hd.m_lanczos_ff;
    h->m_lanczos_nf = hd.m_lanczos_nf;
    h->ichol_relaxer = hd.ichol_relaxer;
    return FSD_OK;
}

int fsd_get_ewald_table(const fsd_handle* h, float* host_table, size_t n_floats) {
    if (!h || !host_table || n_floats < h->ewald_host.size()) return FSD_ERR_BAD_PARAMS;
    memcpy(host_table, h->ewald_host.data(), sizeof(float) * h->ewald_host.size());
    return FSD_OK;
}

int fsd_build_neighbor_list(fsd_handle* h, const float* d_pos) {
    if (!h || !d_pos) return FSD_ERR_BAD_PARAMS;
    for (int attempt = 0; attempt < 3; ++attempt) {
        int maxc = 0;
        FSD_TRY(build_neighbor_list(h, (const float4*)d_pos, &maxc));
        h->info.nlist_max = maxc;
        if (maxc <= h->w.nl_stride) {
            FSD_TRY(build_lub_list(h, (const float4*)d_pos));
            h->nlist_valid = true;
            h->pc_valid = false;
            return FSD_OK;
        }
        // Grow once for the observed count (the only allocation after creation).
        FSD_TRY(alloc_nlist(h, ((maxc * 5 / 4 + 31) / 32) * 32));
    }
    return FSD_ERR_NLIST_OVERFLOW;
}

int fsd_get_neighbor_list(const fsd_handle* h, unsigned int* host_nneigh, unsigned int* host_nlist, size_t cap,
                          int* stride) {
    if (!h || !h->nlist_valid) return FSD_ERR_BAD_PARAMS;
    if (stride) *stride = h->w.nl_stride;
    if (host_nneigh)
        FSD_CHECK_CUDA(cudaMemcpyAsync(host_nneigh, h->w.nneigh, sizeof(unsigned) * h->p.N, cudaMemcpyDeviceToHost,
                                       h->stream));
    if (host_nlist) {
        const size_t need = (size_t)h->p.N * h->w.nl_stride;
        if (cap < need) return FSD_ERR_BAD_PARAMS;
        FSD_CHECK_CUDA(
            cudaMemcpyAsync(host_nlist, h->w.nlist, sizeof(unsigned) * need, cudaMemcpyDeviceToHost, h->stream));
    }
    FSD_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return FSD_OK;
}

int fsd_mobility(fsd_handle* h, const float* d_pos, const float* d_genF, float* d_genU, int parts) {
    if (!h || !d_pos || !d_genF || !d_genU || parts < 1 || parts > 3) return FSD_ERR_BAD_PARAMS;
    if ((parts & 2) && !h->nlist_valid) return FSD_ERR_BAD_PARAMS;
    return mobility_apply(h, (const float4*)d_pos, d_genF, d_genU, parts, nullptr, true);
}

int fsd_lub_rfu(fsd_handle* h, const float* d_pos, const float* d_U6, float* d_F6) {
    if (!h || !h->nlist_valid || !d_pos || !d_U6 || !d_F6) return FSD_ERR_BAD_PARAMS;
    lub_rfu(h, (const float4*)d_pos, d_U6, d_F6, nullptr);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

int fsd_lub_rfe(fsd_handle* h, const float* d_pos, float shear_rate, const float* d_ori, const float* d_b2_mask,
                float B2, float* d_F6) {
    if (!h || !h->nlist_valid || !d_pos || !d_F6) return FSD_ERR_BAD_PARAMS;
    lub_rfe(h, (const float4*)d_pos, shear_rate, (const float3*)d_ori, d_b2_mask, B2, d_F6);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

int fsd_lub_rsu(fsd_handle* h, const float* d_pos, const float* d_U6, float* d_S5) {
    if (!h || !h->nlist_valid || !d_pos || !d_U6 || !d_S5) return FSD_ERR_BAD_PARAMS;
    lub_rsu(h, (const float4*)d_pos, d_U6, d_S5);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

int fsd_lub_rse(fsd_handle* h, const float* d_pos, float shear_rate, const float* d_ori, const float* d_b2_mask,
                float B2, float* d_S5) {
    if (!h || !h->nlist_valid || !d_pos || !d_S5) return FSD_ERR_BAD_PARAMS;
    lub_rse(h, (const float4*)d_pos, shear_rate, (const float3*)d_ori, d_b2_mask, B2, d_S5);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

int fsd_saddle_multiply(fsd_handle* h, const float* d_pos, const float* d_x, float* d_b) {
    if (!h || !h->nlist_valid || !d_pos || !d_x || !d_b) return FSD_ERR_BAD_PARAMS;
    return saddle_multiply(h, (const float4*)d_pos, d_x, d_b, true);
}

int fsd_precond_build(fsd_handle* h, const float* d_pos) {
    if (!h || !h->nlist_valid || !d_pos) return FSD_ERR_BAD_PARAMS;
    return precond_build(h, (const float4*)d_pos);
}

int fsd_precond_set_blocks(fsd_handle* h, int nnzb, const int* d_rowptr, const int* d_col, const float* d_blocks) {
    if (!h || !d_rowptr || (nnzb > 0 && (!d_col || !d_blocks))) return FSD_ERR_BAD_PARAMS;
    return learned_set_blocks(h, nnzb, d_rowptr, d_col, d_blocks);
}

int fsd_learned_num_weights(void) { return MpLayout::total; }

int fsd_learned_set_weights(fsd_handle* h, const float* host_w, int n) {
    if (!h || !host_w) return FSD_ERR_BAD_PARAMS;
    return learned_set_weights(h, host_w, n);
}

int fsd_learned_get_weights(fsd_handle* h, float* host_w, int n) {
    if (!h || !host_w) return FSD_ERR_BAD_PARAMS;
    return mpnn_get_weights(h, host_w, n);
}

int fsd_learned_get_state(fsd_handle* h, float* host, int n, int* adam_step) {
    if (!h || !host || !adam_step) return FSD_ERR_BAD_PARAMS;
    return mpnn_get_state(h, host, n, adam_step);
}

int fsd_learned_set_state(fsd_handle* h, const float* host, int n, int adam_step) {
    if (!h || !host) return FSD_ERR_BAD_PARAMS;
    const int e = mpnn_set_state(h, host, n, adam_step);
    if (e == FSD_OK) learned(h)->g_user = false;
    return e;
}

int fsd_learned_tensor_cores(fsd_handle* h, int on) {
    if (!h) return FSD_ERR_BAD_PARAMS;
    mpnn_use_umma(h, on != 0);
    return FSD_OK;
}

int fsd_learned_set_poly(fsd_handle* h, const float* host_c, int k) {
    if (!h) return FSD_ERR_BAD_PARAMS;
    return poly_set_coefficients(h, host_c, k);
}

int fsd_learned_set_interval(fsd_handle* h, float rho) {
    if (!h || !(rho >= 0.f && rho < 1.f)) return FSD_ERR_BAD_PARAMS;
    LearnedState* s = learned(h);
    s->user_ratio = rho > 0.f ? rho : -1.f;
    if (rho > 0.f) s->poly_user = false;
    return FSD_OK;
}

int fsd_learned_interval_coefficients(float rho, float lambda, int k, float* host_c) {
    if (!host_c || k < 2 || k > kMaxPoly || !(rho > 0.f && rho < 1.f) || !(lambda > 0.f)) return FSD_ERR_BAD_PARAMS;
    poly_interval_coefficients(rho, lambda, k, host_c);
    return FSD_OK;
}

int fsd_learned_ratio_train_step(fsd_handle* h, const float* d_pos, float target_log_ratio, float lr, float* loss,
                                 float* predicted_log_ratio, float* host_grad) {
    if (!h || !d_pos || !h->nlist_valid || h->p.learned_poly < 2) return FSD_ERR_BAD_PARAMS;
    return mpnn_ratio_train_step(h, (const float4*)d_pos, target_log_ratio, lr, loss, predicted_log_ratio,
                                 host_grad);
}

int fsd_learned_get_poly(fsd_handle* h, float* host_c, int n) {
    if (!h) return FSD_ERR_BAD_PARAMS;
    return poly_get_coefficients(h, host_c, n);
}

int fsd_learned_poly_train_step(fsd_handle* h, const float* d_pos, int n_probes, unsigned int step, float lr,
                                int natural, float* loss, float* loss_opt, float* host_grad, float* host_coef,
                                float* host_coef_opt) {
    if (!h || !d_pos || !h->nlist_valid || n_probes < 1 || n_probes > 64) return FSD_ERR_BAD_PARAMS;
    const int k = h->p.learned_poly;
    if (k < 2) return FSD_ERR_BAD_PARAMS;
    return mpnn_poly_train_step(h, (const float4*)d_pos, n_probes, step, lr, k, natural, loss, loss_opt, host_grad,
                                host_coef, host_coef_opt);
}

int fsd_learned_train_step(fsd_handle* h, const float* d_pos, const float* host_probes, int n_probes,
                           unsigned int step, float lr, float* loss, float* host_grad) {
    if (!h || !d_pos || !h->nlist_valid || n_probes < 1) return FSD_ERR_BAD_PARAMS;
    return mpnn_train_step(h, (const float4*)d_pos, host_probes, n_probes, step, lr, loss, host_grad);
}

int fsd_precond_apply(fsd_handle* h, const float* d_b, float* d_x) {
    if (!h || !h->pc_valid || !d_b || !d_x) return FSD_ERR_BAD_PARAMS;
    // Some applications gather b from neighbouring particles while writing x
    // (the approximate inverse applied once), so overlapping vectors go
    // through a copy.  The saddle work vector is free outside a solve.
    const size_t n17 = 17 * (size_t)h->p.N;
    const bool overlap = d_b < d_x + n17 && d_x < d_b + n17;
    if (overlap) {
        FSD_CHECK_CUDA(cudaMemcpyAsync(h->w.sz, d_b, sizeof(float) * n17, cudaMemcpyDeviceToDevice, h->stream));
        d_b = h->w.sz;
    }
    return precond_apply(h, d_b, d_x);
}

int fsd_saddle_solve(fsd_handle* h, const float* d_pos, const float* d_rhs, float* d_x, int* iters, float* resid) {
    if (!h || !h->nlist_valid || !h->pc_valid || !d_pos || !d_rhs || !d_x) return FSD_ERR_BAD_PARAMS;
    int it = 0;
    float rs = 0;
    const int st = saddle_solve(h, (const float4*)d_pos, d_rhs, d_x, h->p.solver_tol, &it, &rs);
    h->info.gmres_iters[2] = it;
    h->info.gmres_resid[2] = rs;
    h->info.status = st;
    if (iters) *iters = it;
    if (resid) *resid = rs;
    return st;
}

}  // extern "C"
