// Host harness around the reference's own device functions and set-up blocks.
//
// Test infrastructure only: compiled by build_ref.py into oracle/_ref/libfsdref.so
// and loaded by the tests (through oracle/refbind.py) to produce reference outputs.
// Every exported function runs one extracted reference kernel over all threads of
// its launch, one thread at a time, with an identity group-member array.
#include "hoomd_shim.h"
#include <string>
using std::abs;
using std::max;
using std::min;

#define SINGLE_PRECISION 1
#define __scalar2int_rd __float2int_rd

#include "extracted_kernels.inc"

void genrcm(int node_num, int adj_num, int adj_row[], int adj[], int perm[]);

namespace {
std::vector<unsigned> identity(unsigned n) {
    std::vector<unsigned> g(n);
    for (unsigned i = 0; i < n; ++i) g[i] = i;
    return g;
}
template <class F> void launch1d(unsigned n, F&& f) {
    blockDim = dim3(1, 1, 1);
    threadIdx = dim3(0, 0, 0);
    for (unsigned i = 0; i < n; ++i) {
        blockIdx = dim3(i, 0, 0);
        f();
    }
}

struct StokesSetup {
    Scalar m_xi, m_error, m_max_strain;
    Scalar m_ewald_cut = 0, m_ewald_dr = 0;
    int m_ewald_n = 0;
    int m_Nx = 0, m_Ny = 0, m_Nz = 0, m_gaussP = 0;
    Scalar m_gaussm = 0, m_eta = 0;
    Scalar3 m_gridh{0, 0, 0};
    Scalar2 m_self{0, 0};
    GPUArray<Scalar4> m_ewaldC1;
    ExecConf* m_exec_conf = nullptr;
    struct PData {
        BoxDim box;
        const BoxDim& getBox() const { return box; }
    } pdata;
    PData* m_pdata = &pdata;
    void grid() {
#include "setparams_grid.inc"
    }
    void ewald() {
#include "setparams_ewald.inc"
    }
};
}  // namespace

extern "C" {

// Stokes::setParams grid/support selection.  out_i = {Nx, Ny, Nz, P};
// out_f = {rcut, gaussm, eta, hx, hy, hz}.
int ref_setparams(float xi, float error, float max_strain, float Lx, float Ly, float Lz,
                  int* out_i, float* out_f) {
    StokesSetup s;
    s.m_xi = xi; s.m_error = error; s.m_max_strain = max_strain;
    s.pdata.box = BoxDim(Lx, Ly, Lz, 0);
    s.grid();
    out_i[0] = s.m_Nx; out_i[1] = s.m_Ny; out_i[2] = s.m_Nz; out_i[3] = s.m_gaussP;
    out_f[0] = s.m_ewald_cut; out_f[1] = s.m_gaussm; out_f[2] = s.m_eta;
    out_f[3] = s.m_gridh.x; out_f[4] = s.m_gridh.y; out_f[5] = s.m_gridh.z;
    return 0;
}

// Stokes::setParams real-space Ewald table and self terms.  Returns nR; when
// table is non-null it receives 2*nR float4 entries.
int ref_ewald_table(float xi, float error, float* table, float* self2, float* ewald_cut_out, int* ewald_n_out) {
    StokesSetup s;
    s.m_xi = xi; s.m_error = error; s.m_max_strain = 0.5f;
    s.m_ewald_cut = sqrtf(-logf(error)) / xi;
    s.ewald();
    int nR = s.m_ewald_n + 1;
    if (table) memcpy(table, s.m_ewaldC1.v.data(), sizeof(Scalar4) * 2 * nR);
    self2[0] = s.m_self.x; self2[1] = s.m_self.y;
    *ewald_cut_out = s.m_ewald_cut;
    *ewald_n_out = s.m_ewald_n;
    return nR;
}

void ref_gridk(Scalar4* gridk, int Nx, int Ny, int Nz, float Lx, float Ly, float Lz, float xy, float xi, float eta) {
    BoxDim box(Lx, Ly, Lz, xy);
    unsigned G = Nx * Ny * Nz;
    launch1d(G, [&] { Mobility_SetGridk_kernel(gridk, Nx, Ny, Nz, G, box, xi, eta); });
}

// grids: 11 consecutive complex grids of G points, ordered X Y Z XX XY XZ YX YY YZ ZX ZY.
void ref_green(Scalar2* grids, Scalar4* gridk, unsigned G) {
    Scalar2* g[11];
    for (int i = 0; i < 11; ++i) g[i] = grids + (size_t)i * G;
    launch1d(G, [&] {
        Mobility_WaveSpace_Green_kernel(g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], g[9], g[10], gridk, G);
    });
}

void ref_ts2c(Scalar4* couplet, Scalar4* ts, unsigned N) {
    launch1d(N, [&] { Mobility_TS2C_kernel(couplet, ts, N); });
}
void ref_d2we(Scalar4* delu, Scalar4* omegaE, unsigned N) {
    launch1d(N, [&] { Mobility_D2WE_kernel(delu, omegaE, N); });
}

void ref_realspace(Scalar4* pos, Scalar4* vel, Scalar4* delu, Scalar4* force, Scalar4* couplet, int N, float xi,
                   Scalar4* table, float self_x, float self_y, float ewald_cut, int ewald_n, float ewald_dr,
                   float Lx, float Ly, float Lz, float xy, const unsigned* nneigh, const unsigned* nlist,
                   const unsigned* head) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    Scalar2 self{self_x, self_y};
    launch1d(N, [&] {
        Mobility_RealSpace_kernel(pos, vel, delu, force, couplet, N, xi, table, self, ewald_cut, ewald_n, ewald_dr,
                                  gm.data(), box, nneigh, nlist, head);
    });
}

void ref_rfu(float* F, const float* U, const Scalar4* pos, int N, float Lx, float Ly, float Lz, float xy,
             const unsigned* nneigh, unsigned* nlist, const unsigned* head, const float* tdist, const float* tvals,
             float tmin, float tdr, float rlub) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Lubrication_RFU_kernel(F, U, pos, gm.data(), N, box, nneigh, nlist, head, tdist, tvals, tmin, tdr, rlub);
    });
}

void ref_rfe(float* F, float shear_rate, Scalar4* pos, float B2, float* b2mask, Scalar3* ori, int N, float Lx,
             float Ly, float Lz, float xy, const unsigned* nneigh, unsigned* nlist, const unsigned* head,
             const float* tdist, const float* tvals, float tmin, float tdr, float rlub) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Lubrication_RFE_kernel(F, shear_rate, pos, B2, b2mask, ori, gm.data(), N, box, nneigh, nlist, head, tdist,
                               tvals, tmin, tdr, rlub);
    });
}

void ref_rsu(float* S, float* U, Scalar4* pos, int N, float Lx, float Ly, float Lz, float xy, const unsigned* nneigh,
             unsigned* nlist, const unsigned* head, const float* tdist, const float* tvals, float tmin, float tdr,
             float rlub) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Lubrication_RSU_kernel(S, U, pos, gm.data(), N, box, nneigh, nlist, head, tdist, tvals, tmin, tdr, rlub);
    });
}

void ref_rse(float* S, float shear_rate, float B2, float* b2mask, Scalar3* ori, int N, const unsigned* nneigh,
             unsigned* nlist, const unsigned* head, Scalar4* pos, float Lx, float Ly, float Lz, float xy,
             const float* tdist, const float* tvals, float tmin, float tdr) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Lubrication_RSE_kernel(S, shear_rate, B2, b2mask, ori, N, gm.data(), nneigh, nlist, head, pos, box, tdist,
                               tvals, tmin, tdr);
    });
}

// Pruned (r < rp) neighbour list, with self, sorted by index: the reference's
// preconditioner graph.  head must have N+1 entries; nlist_p enough room.
void ref_pruned_nlist(const Scalar4* pos, int N, float Lx, float Ly, float Lz, float xy, const unsigned* nneigh,
                      const unsigned* nlist, const unsigned* head, float rp, unsigned* nneigh_p, unsigned* nlist_p,
                      unsigned* head_p, unsigned* nless) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Precondition_GetPrunedNneigh_kernel(nneigh_p, N, pos, box, gm.data(), nneigh, nlist, head, rp);
    });
    head_p[0] = 0;
    for (int i = 0; i < N; ++i) head_p[i + 1] = head_p[i] + nneigh_p[i];
    launch1d(N, [&] {
        Precondition_GetPrunedNlist_kernel(nneigh_p, nlist_p, head_p, nless, N, pos, box, gm.data(), nneigh, nlist,
                                           head, rp);
    });
}

// Pruned R_FU in COO (row, col, val), in the reference's entry order.  Returns nnz.
int ref_precond_rfu_coo(const Scalar4* pos, int N, float Lx, float Ly, float Lz, float xy, unsigned* nneigh_p,
                        unsigned* nlist_p, unsigned* head_p, unsigned* nless, const float* tdist, const float* tvals,
                        float tmin, float tdr, float rp, int* row, int* col, float* val, int cap) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    std::vector<unsigned> nepp(2 * N), offset(N);
    launch1d(N, [&] { Precondition_NEPP_kernel(N, gm.data(), nneigh_p, nlist_p, head_p, nepp.data()); });
    offset[0] = 0;
    for (int i = 1; i < N; ++i) offset[i] = offset[i - 1] + nepp[i - 1] + nepp[N + i - 1];
    int nnz = offset[N - 1] + nepp[N - 1] + nepp[2 * N - 1];
    if (nnz > cap) return -nnz;
    memset(val, 0, sizeof(float) * nnz);
    launch1d(N, [&] {
        Precondition_RFU_kernel(N, gm.data(), nneigh_p, nless, nlist_p, head_p, nepp.data(), offset.data(),
                                const_cast<Scalar4*>(pos), box, tdist, tvals, tmin, tdr, row, col, val, rp);
    });
    return nnz;
}

void ref_add_identity(float* val, int* rowptr, int* colind, int N, float relaxer) {
    launch1d(N, [&] { Precondition_AddIdentity_kernel(val, rowptr, colind, N, relaxer); });
}

void ref_setforce(const Scalar4* pos, Scalar3* ori, float* F, int N, const unsigned* nneigh, unsigned* nlist,
                  const unsigned* head, float ndsr, float k_n, float kappa, float beta, float epsq, float T_ext,
                  float Lx, float Ly, float Lz, float xy) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Stokes_SetForce_manually_kernel(pos, ori, F, N, gm.data(), nneigh, nlist, head, ndsr, k_n, kappa, beta, epsq,
                                        T_ext, box);
    });
}

void ref_add_strain_rate(float* b, float shear_rate, float B2, float* b2mask, Scalar3* ori, unsigned N) {
    auto gm = identity(N);
    launch1d(N, [&] { Integrator_AddStrainRate_kernel(b, shear_rate, gm.data(), B2, b2mask, ori, N); });
}

void ref_euler(Scalar4* pos_in, Scalar4* pos_out, float* vel, int3* image, unsigned N, float Lx, float Ly, float Lz,
               float xy, float dt) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] { Integrator_ExplicitEuler_kernel(pos_in, pos_out, vel, image, gm.data(), N, box, dt); });
}

void ref_euler_shear(Scalar4* pos, Scalar3* ori, Scalar4* pos_gb, float* vel, float B1, float* b1mask,
                     Scalar3* noise_ang, int3* image, unsigned N, float Lx, float Ly, float Lz, float xy, float dt,
                     float shear_rate) {
    BoxDim box(Lx, Ly, Lz, xy);
    auto gm = identity(N);
    launch1d(N, [&] {
        Integrator_ExplicitEuler_Shear_kernel(pos, ori, pos, ori, pos_gb, vel, B1, b1mask, noise_ang, image, gm.data(),
                                              N, box, dt, shear_rate);
    });
}

void ref_rng_grid(Scalar2* grids, Scalar4* gridk, float* gauss2, int Nx, int Ny, int Nz, float T, float dt,
                  float quadW) {
    unsigned G = Nx * Ny * Nz;
    Scalar2* g[11];
    for (int i = 0; i < 11; ++i) g[i] = grids + (size_t)i * G;
    launch1d(G, [&] {
        Brownian_FarField_RNG_Grid1of2_kernel(g[0], g[1], g[2], gridk, gauss2, G, Nx, Ny, Nz, 0u, T, dt, quadW);
    });
    launch1d(G, [&] {
        Brownian_FarField_RNG_Grid2of2_kernel(g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], g[9], g[10],
                                              gridk, G);
    });
}

// genrcm from the reference's vendored rcm.cpp (1-based CSR adjacency in, 1-based permutation out).
void ref_genrcm(int node_num, int adj_num, int* adj_row, int* adj, int* perm) {
    genrcm(node_num, adj_num, adj_row, adj, perm);
}

}  // extern "C"
