/*
 * fsd.h -- C ABI of the B200 Fast Stokesian Dynamics velocity path.
 *
 * A drop-in for the deterministic + Brownian velocity path of the PSEv3
 * HOOMD-blue plugin (GeZhouyang/FSD).  Every entry point takes plain device
 * pointers and sizes; no C++ or torch types cross this boundary.  Pointers
 * named d_* are device pointers and are borrowed: the caller owns them.  All
 * work is enqueued on the stream given to fsd_create (or fsd_set_stream);
 * entry points that report a solver outcome synchronise that stream.
 *
 * Data layouts follow the reference exactly (DataStruct.h, Stokes.h:189-190):
 *   positions      float4 x N   (x, y, z, unused), box centred on the origin
 *   orientations   float3 x N
 *   images         int3   x N
 *   generalized force  (11N): [F_i, L_i] (6 per particle) then S_i (5 per particle)
 *   generalized velocity (11N): [U_i, W_i] then E_i, same ordering
 *   stresslet / strain order: (xx-zz, 2xy, 2xz, 2yz, yy-zz) for strain,
 *                             (Sxx, Sxy, Sxz, Syz, Syy) for stresslets
 *   saddle vectors (17N): [F^ff (6N) | S^ff (5N) | U - U_inf (6N)]
 *
 * Errors: every function returns an fsd_status.  Nothing calls exit().
 * Threading: a handle is not re-entrant; use one handle per host thread.
 */
#ifndef FSD_H
#define FSD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fsd_handle fsd_handle;

enum fsd_status {
    FSD_OK = 0,
    FSD_ERR_BAD_PARAMS = 1,     /* parameters the reference rejects with exit() (Stokes.cc:140-261) */
    FSD_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    FSD_ERR_GMRES_MAXIT = 3,    /* GMRES hit its iteration limit (Solvers.cu:121) or stayed above its
                                   tolerance after restarting from the true residual */
    FSD_ERR_LANCZOS_MAXIT = 4,  /* Lanczos did not reach its tolerance (Brownian_FarField.cu:787) */
    FSD_ERR_ICHOL = 5,          /* incomplete Cholesky failed even after relaxation (Precondition.cu:1246) */
    FSD_ERR_NLIST_OVERFLOW = 6, /* more neighbours than the list capacity even after growing it */
    FSD_ERR_DEVICE_WAIT = 7,    /* a bounded device-side wait ran out */
    FSD_ERR_ALLOC = 8,          /* device allocation failed */
    FSD_ERR_BREAKDOWN = 9       /* Krylov breakdown or a non-finite value */
};

enum fsd_precond_kind {
    FSD_PRECOND_NONE = 0,    /* identity (Saddle.cu:258 debug path) */
    FSD_PRECOND_ICHOL = 1,   /* block preconditioner with RCM + IC(0) of pruned R_FU (Saddle.cu:171) */
    FSD_PRECOND_LEARNED = 2  /* learned block-sparse approximate inverse of the same block */
};

enum fsd_force_mode {
    FSD_FORCE_INTERPARTICLE = 0, /* overwrite applied force with the built-in pair force (Helper_Stokes.cu:65) */
    FSD_FORCE_USER = 1           /* keep the caller's applied force/torque untouched */
};

/* Integrator parameters.  Defaults (fsd_default_params) are the reference
 * defaults of PSEv3.__init__ (integrate.py:40-55). */
typedef struct fsd_params {
    int N;                       /* number of particles (radius a = 1) */
    float Lx, Ly, Lz, xy;        /* box edges and xy tilt */
    float xi;                    /* Ewald splitting parameter (0.5) */
    float error;                 /* Ewald / spreading accuracy (1e-3) */
    float max_strain;            /* maximum box strain, widens the Gaussian support (0.5) */
    float solver_tol;            /* GMRES relative residual; the reference uses `error` (Stokes.cc:1449) */
    float lanczos_tol;           /* Lanczos relative change; the reference uses `error` */
    float rfd_epsilon;           /* random finite difference step; the reference uses `error` (Stokes.cc:125) */
    float T;                     /* temperature kT */
    float dt;                    /* time step */
    uint32_t seed;               /* random seed (hashed as Stokes.cc:74) */
    float ndsr, kappa, k_n, beta_AF, epsq;  /* pair force (integrate.py:54) */
    float T_ext, omega_ext;      /* external torque amplitude and frequency */
    float sqm_B1, sqm_B2;        /* squirmer modes */
    int N_mix;                   /* particles with tag < N_mix keep the unmasked modes */
    float coef_B1_mask, coef_B2_mask;
    float rot_diff;              /* rotational diffusivity of the director noise */
    int period;                  /* stresslet output period (0 = never) */
    int gmres_restart;           /* 50 (Solvers.cu:105) */
    int gmres_max_iter;          /* 1000 (Solvers.cu:117) */
    int lanczos_max;             /* 100 (Brownian_FarField.cu:618) */
    int precond;                 /* fsd_precond_kind */
    int force_mode;              /* fsd_force_mode */
    int kgrid_pi_ref;            /* 1: wave vectors scaled by 2*3.1416926536 as Helper_Mobility.cu:389; 0: 2*pi */
    float rlub;                  /* lubrication cutoff (4.0, Stokes.cc:1505) */
    float rp;                    /* preconditioner cutoff (2.1, Stokes.cc:1506) */
    float nlist_buffer;          /* neighbour-list skin added to the Ewald cutoff (0.4, integrate.py:83) */
    int ichol_local_shift;       /* 1: shift only failing IC(0) pivot blocks (default); 0: double the global
                                    relaxer and refactor, as Precondition.cu:1457-1489 */
    float ichol_gain_limit;      /* largest accepted relaxer * lambda_max(G) of the IC(0) inverse, estimated by
                                    power iteration after each factorisation; above it the relaxer doubles and
                                    the factor is rebuilt (100; 0 = no check).  The exact (R + relaxer D)^-1
                                    has relaxer * lambda_max <= 1. */
    int learned_inner;           /* FSD_PRECOND_LEARNED: inner GMRES steps on R_FU^pruned + D per application,
                                    right-preconditioned by the learned block-sparse G (4; 0 = apply G once).
                                    With inner steps the outer solve is flexible GMRES. */
    int learned_poly;            /* FSD_PRECOND_LEARNED: when >= 2 (at most 16), y ~ (R_FU^pruned + D)^-1 t is
                                    G q(AG) t with a polynomial q of degree learned_poly - 1, expanded in
                                    Chebyshev polynomials on [0, lambda] (lambda: power-iteration bound of
                                    the spectrum of AG, times 1.1), so 1 - x q(x) is the Chebyshev
                                    acceleration on [rho lambda, lambda]; the network predicts rho for each
                                    configuration.  The outer solve stays plain GMRES.  0 (default):
                                    learned_inner decides. */
    float poly_interval;         /* learned_poly without network weights: the fixed ratio rho (0.05); 0 = fit
                                    the coefficients to four probe vectors at every build instead */
    int autotune;                /* 1: time candidate spreading tiles and FFT line batches on the first mobility
                                    call and keep the fastest (cached per process and grid shape).  Results then
                                    depend on the choice through the summation order, so runs in different
                                    processes may differ in the last bits.  0 (default): fixed shapes. */
    int friction_type;           /* 0: none (default); 1: TYPE1, the frictional contact terms added to the
                                    tabulated YA, YB, YC functions for gaps h <= friction_h0
                                    (Stokes::setFriction, Stokes.cc:1132-1191) */
    float friction_h0;           /* largest gap with frictional contact */
    float friction_alpha[6];     /* strengths for YA11, YA12, YB11, YB12, YC11, YC12 */
    int integrator;              /* 0: explicit Euler (Integrator_ExplicitEuler_Shear_kernel, the live path);
                                    1: two-stage Runge-Kutta (Heun) of Integrator.cu:232-438, which evaluates
                                    the velocity again at the Euler predictor with the same step's draws */
} fsd_params;

/* Derived PSE parameters (Stokes::setParams, Stokes.cc:118-696). */
typedef struct fsd_pse_info {
    int Nx, Ny, Nz, P;
    float ewald_cut, gauss_m, eta, hx, hy, hz;
    float self_x, self_y;
    int ewald_n;
    float ewald_dr;
} fsd_pse_info;

/* Outcome of the last solve or step. */
typedef struct fsd_solve_info {
    int gmres_iters[3];          /* RFD forward, RFD backward, main solve */
    float gmres_resid[3];        /* final relative residual ||b - Ax|| / ||b|| */
    int lanczos_ff_iters, lanczos_nf_iters;
    float lanczos_ff_err, lanczos_nf_err;
    int ichol_attempts;          /* factorisations tried (relaxer doubled after each failure) */
    float ichol_relaxer;         /* relaxer the factorisation succeeded with */
    int nlist_max;               /* largest neighbour count seen */
    int status;                  /* fsd_status of that call */
    int ichol_shifted;           /* pivot blocks that needed a local shift */
    float ichol_gain;            /* power-iteration estimate of lambda_max(G) of the accepted factor */
    int poly_source;             /* learned_poly: coefficients of the last build, 1 the Chebyshev interval the
                                    network predicts, 2 a least-squares fit on probe vectors, 3 the caller's,
                                    4 a fixed interval (0: not in use) */
    float poly_loss_net;         /* probe loss ||t - AG q(AG) t||^2/||t||^2 of the network's coefficients at
                                    the last build (-1: none) */
    float poly_loss_fit;         /* loss of the least-squares fit on its four probes (-1: not fitted) */
    float poly_ratio;            /* Chebyshev interval ratio rho of the last build (-1: none) */
} fsd_solve_info;

/* Arguments of one time step (Stokes_StepOne, Stokes.cuh:81-108). */
typedef struct fsd_step_args {
    unsigned int timestep;
    float shear_rate;            /* current shear rate (ShearFunction::getShearRate) */
    float* d_pos;                /* float4 x N, in/out */
    float* d_ori;                /* float3 x N, in/out */
    float* d_pos_gb;             /* float4 x N, unwrapped positions, in/out (may be NULL) */
    int* d_image;                /* int3 x N, in/out */
    float* d_force;              /* 6N applied force/torque; written when force_mode = INTERPARTICLE */
    float* d_velocity;           /* 11N out: [U, W] (6N) then stresslet (5N, on output steps) */
    const float* d_noise_ang;    /* float3 x N angular noise, or NULL for none */
    const float* d_b1_mask;      /* N floats, or NULL for all ones */
    const float* d_b2_mask;      /* N floats, or NULL for all ones */
} fsd_step_args;

void fsd_default_params(fsd_params* p);
const char* fsd_status_string(int status);

/* Host-only part of Stokes::setParams (Stokes.cc:118-696): grid, support,
 * splitting and the real-space Ewald table (2*(ewald_n+1) float4, written to
 * host_table when it is non-NULL and n_floats is large enough).  Touches no
 * GPU. */
int fsd_pse_setup(const fsd_params* p, fsd_pse_info* info, float* host_table, size_t n_floats);

/* The tabulated near-field resistance functions a handle with these
 * parameters uses: dist (1000 floats) and vals (1000 x 22 floats), with the
 * friction patch of Stokes::setFriction (Stokes.cc:1132-1191) applied when
 * friction_type is 1.  Host only. */
int fsd_resistance_table(const fsd_params* p, float* dist, float* vals);

/* Reverse Cuthill-McKee ordering of an n-node graph given as 0-based CSR
 * adjacency (rows may include self loops); perm[new] = old.  Replaces the
 * host genrcm call of the preconditioner (rcm.cpp:1009, Precondition.cu:1009)
 * and returns the same ordering.  Host only. */
int fsd_rcm_order(int n, const int* rowptr, const int* col, int* perm);

/* Stokes constructor + setParams + setResistanceTable + setSparseMath +
 * AllocateWorkSpaces (Stokes.cc:47-83, 118-696, 937-1063;
 * Stokes_ResistanceTable.cc:33; Stokes_SparseMath.cc:15).  All device memory
 * the path needs is allocated here; nothing is allocated per step. */
int fsd_create(const fsd_params* p, void* cuda_stream, fsd_handle** out);
/* Stokes destructor (Stokes.cc:86-113). */
void fsd_destroy(fsd_handle* h);
int fsd_set_stream(fsd_handle* h, void* cuda_stream);
/* Number of CUDA kernels this library has launched since it was loaded (no
 * counterpart in the reference; used to report launches per step). */
unsigned long long fsd_launch_count(void);
/* Box update (HOOMD box_resize with shear_variant, variant.py:14-32). */
int fsd_set_box(fsd_handle* h, float Lx, float Ly, float Lz, float xy);
/* Stokes::setT / temperature variant value for the next step. */
int fsd_set_temperature(fsd_handle* h, float T);
int fsd_get_pse_info(const fsd_handle* h, fsd_pse_info* info);
/* Per-region device timing with CUDA events (no counterpart in the reference,
 * whose only timing is HOOMD's profiler around the whole step, Stokes.cc:1201).
 * Regions, in order: neighbour list, preconditioner build, spread, FFT,
 * Green, contract, real space, R_FU, preconditioner apply, Krylov vector ops,
 * Lanczos vector ops, wave-space noise, other lubrication, integration.
 * fsd_profile_read fills ms[] and counts[] (n >= 14) and optionally resets;
 * with n >= 15, counts[14] receives the number of regions left untimed
 * because no CUDA event could be created (0 in normal operation). */
int fsd_profile_enable(fsd_handle* h, int on);
int fsd_profile_read(fsd_handle* h, double* ms, long long* counts, int n, int reset);
int fsd_get_solve_info(const fsd_handle* h, fsd_solve_info* info);

/* Checkpoint of the solver state one step carries into the next (the carried
 * state of Stokes::integrateStepOne, Stokes.cc:1658-1666, and the main
 * solve's warm start, Integrator.cu:777): the saddle solution (17N floats),
 * the far- and near-field Lanczos sizes and the IC(0) relaxer.  Positions,
 * orientations, images and the timestep are the caller's; the Brownian
 * draws are keyed by (seed, timestep), so a handle created with the same
 * parameters, loaded from a checkpoint and given the same caller arrays
 * continues the trajectory bit for bit.  fsd_checkpoint_size gives the
 * bytes; save writes them to host memory, load reads them back (same N;
 * FSD_ERR_BAD_PARAMS for a checkpoint of another size or format). */
size_t fsd_checkpoint_size(const fsd_handle* h);
int fsd_checkpoint_save(fsd_handle* h, void* host, size_t bytes);
int fsd_checkpoint_load(fsd_handle* h, const void* host, size_t bytes);
/* Copy the real-space Ewald table (2*(ewald_n+1) float4) to host memory. */
int fsd_get_ewald_table(const fsd_handle* h, float* host_table, size_t n_floats);

/* Full neighbour list within ewald_cut + buffer (replaces HOOMD
 * NeighborListGPUBinned, integrate.py:80-85, computed at Stokes.cc:1216).
 * Must precede the pair entry points below for the same positions. */
int fsd_build_neighbor_list(fsd_handle* h, const float* d_pos);
/* Copy the list to host: counts (N), and row entries (N x stride). */
int fsd_get_neighbor_list(const fsd_handle* h, unsigned int* host_nneigh, unsigned int* host_nlist,
                          size_t cap, int* stride);

/* Neighbour list that allocates nothing.  No counterpart in the reference.
 *
 * fsd_create allocates the handle's device workspaces, and some callers
 * cannot do that at the point where they need a list: an integrator whose
 * host application owns all device memory through its own pool and gives a
 * plug-in none of its own, or a step loop in which cudaMalloc/cudaFree,
 * which can synchronise the whole device, are not allowed.  This entry point
 * takes only the caller's buffers and does its cell binning in one fixed
 * file-scope device array of about 1.25 MiB that every GPU loading the
 * library holds until the process exits.
 *
 * Same lists as fsd_build_neighbor_list with r_list = ewald_cut + buffer:
 * for each particle, every j != i with |minImage(x_i - x_j)|^2 < rlist^2, in
 * a deterministic (not sorted) order.  d_pos: float4 x N; d_nneigh: N counts;
 * d_nlist: N x stride entries; *d_max_count (device int) receives the
 * largest count before capping: a value above stride means rows were
 * truncated and the call should be repeated with a larger stride.
 * N above FSD_NOALLOC_MAX_N, stride < 1, a non-positive box length or rlist
 * return FSD_ERR_BAD_PARAMS before any GPU work.  Boxes whose cell grid
 * would exceed FSD_NOALLOC_MAX_CELLS use fewer, wider cells.
 *
 * The first call on each device looks up the array's device address (with
 * that device current); make that first call before any stream capture.
 * The address is kept for the life of the process: after cudaDeviceReset (or
 * anything else that destroys the device's primary context) it is stale, so
 * do not call this entry point on a device that was reset.
 * All calls on a device share the array: calls whose GPU work overlaps
 * (different streams without ordering between them) race and corrupt each
 * other's lists.  Order them on one stream or with events. */
#define FSD_NOALLOC_MAX_N 65536
#define FSD_NOALLOC_MAX_CELLS 65536
int fsd_neighbor_list_noalloc(const float* d_pos, int N, float Lx, float Ly, float Lz, float xy, float rlist,
                              unsigned int* d_nneigh, unsigned int* d_nlist, int stride, int* d_max_count,
                              void* cuda_stream);

/* Generalized far-field mobility U = M^ff F on 11N vectors
 * (Mobility_GeneralizedMobility, Mobility.cu:1488).  parts: 1 = wave space
 * only, 2 = real space + self only, 3 = both (the reference). */
int fsd_mobility(fsd_handle* h, const float* d_pos, const float* d_genF, float* d_genU, int parts);

/* Lubrication pair products over the neighbour list (Lubrication.cu). */
int fsd_lub_rfu(fsd_handle* h, const float* d_pos, const float* d_U6, float* d_F6);          /* F = R_FU U (:69) */
int fsd_lub_rfe(fsd_handle* h, const float* d_pos, float shear_rate, const float* d_ori,
                const float* d_b2_mask, float B2, float* d_F6);                               /* F += R_FE:E (:350) */
int fsd_lub_rsu(fsd_handle* h, const float* d_pos, const float* d_U6, float* d_S5);          /* S -= R_SU U (:650) */
int fsd_lub_rse(fsd_handle* h, const float* d_pos, float shear_rate, const float* d_ori,
                const float* d_b2_mask, float B2, float* d_S5);                               /* S += R_SE:E (:953) */

/* Saddle-point operator b = A x on 17N vectors (Saddle_Multiply, Saddle.cu:80). */
int fsd_saddle_multiply(fsd_handle* h, const float* d_pos, const float* d_x, float* d_b);
/* Build the near-field preconditioner for these positions (Precondition_Wrap, Precondition.cu:1326). */
int fsd_precond_build(fsd_handle* h, const float* d_pos);
/* Set the block-sparse G used by FSD_PRECOND_LEARNED in place of the IC(0)
 * factor's (L L^T)^-1 inside the saddle preconditioner (Saddle.cu:171-264;
 * the explicit-G slot itself has no counterpart in the reference).  Block CSR
 * over particles in their original order: d_rowptr (N+1), d_col (nnzb),
 * d_blocks (nnzb x 36, row-major 6x6 fp32).  The structure is checked
 * (rowptr monotone, rowptr[N] = nnzb, 0 <= col < N) and the arrays copied. */
int fsd_precond_set_blocks(fsd_handle* h, int nnzb, const int* d_rowptr, const int* d_col, const float* d_blocks);
/* Learned preconditioner (FSD_PRECOND_LEARNED; no counterpart in the
 * reference, which factors the same block by IC(0)).  G ~ (R_FU^pruned + D)^-1
 * is the sparse approximate inverse of that matrix on the two-hop sets of the
 * pruned contact graph (FP64 least squares per particle), plus, once weights
 * are set, a correction predicted by a message-passing network on the same
 * pairs from rotation-invariant pair features through an axisymmetric 6x6
 * block basis (so G rotates with the configuration).  Weights are one flat
 * fp32 vector of fsd_learned_num_weights() entries (layout in
 * fsd_b200/csrc/fsd_mpnn.h); blocks set with fsd_precond_set_blocks replace
 * both until weights are set again.
 * fsd_learned_train_step: loss E_z ||A G z - z||^2 / 6N over n_probes probe
 * vectors z (host_probes, n_probes x 6N; or NULL for z = w - A G0 w, the
 * residuals the uncorrected approximate inverse G0 leaves for counter-based
 * normals w drawn from (seed, step)), its gradient (host_grad, optional)
 * and, when lr > 0, one Adam step.  The neighbour list must be current for d_pos.
 * fsd_learned_tensor_cores(h, 0) runs the dense layers in FP32 SIMT instead
 * of BF16 on the tensor cores. */
int fsd_learned_num_weights(void);
int fsd_learned_set_weights(fsd_handle* h, const float* host_w, int n);
int fsd_learned_get_weights(fsd_handle* h, float* host_w, int n);
int fsd_learned_tensor_cores(fsd_handle* h, int on);
/* Training state: weights, Adam first and second moments (3 x num_weights
 * floats) and the Adam step count, to continue training on another handle. */
int fsd_learned_get_state(fsd_handle* h, float* host, int n, int* adam_step);
int fsd_learned_set_state(fsd_handle* h, const float* host, int n, int adam_step);
int fsd_learned_train_step(fsd_handle* h, const float* d_pos, const float* host_probes, int n_probes,
                           unsigned int step, float lr, float* loss, float* host_grad);
/* Learned inner polynomial (learned_poly >= 2; no counterpart in the
 * reference).  fsd_learned_set_poly fixes the k Chebyshev coefficients c of
 * q (k = learned_poly, 2..16) instead of the network's prediction, until
 * weights are set again; fsd_learned_get_poly copies the coefficients in use
 * and, at index 16, the spectral bound lambda of AG of the last build
 * (n >= 17 floats).
 * fsd_learned_poly_train_step: for this configuration (neighbour list current
 * for d_pos), the loss E_t ||t - AG q(AG) t||^2 / ||t||^2 over n_probes
 * (1..64) normal probe vectors drawn from (seed, step), with q's coefficients
 * from the network; its least-squares optimum over all coefficients
 * (loss_opt, host_coef_opt, both optional); the network's coefficients
 * (host_coef, optional, k floats); the weight gradient (host_grad,
 * optional); and, when lr > 0, one Adam step.  With natural != 0 the
 * network is fed the Gauss-Newton direction 2 (c - c_opt) in place of the
 * loss gradient (the loss is quadratic in c with a badly conditioned
 * Hessian); host_grad then holds that direction's weight gradient.
 * These train the coefficients themselves (the loss a least-squares fit
 * minimises); the default learned_poly mode trains the interval instead
 * (fsd_learned_ratio_train_step). */
int fsd_learned_set_poly(fsd_handle* h, const float* host_c, int k);
/* Fixed Chebyshev interval ratio rho (0 < rho < 1) for the next builds in
 * place of the network's prediction (0 clears it; setting weights clears it
 * too), and the coefficients of that interval's polynomial for a spectral
 * bound lambda and k terms (host only). */
int fsd_learned_set_interval(fsd_handle* h, float rho);
int fsd_learned_interval_coefficients(float rho, float lambda, int k, float* host_c);
/* One training step of the interval network on this configuration (the
 * neighbour list current for d_pos): the squared error between the predicted
 * log rho and target_log_ratio (the ratio that gave the fewest outer
 * iterations), the prediction, the weight gradient (host_grad, optional,
 * fsd_learned_num_weights() floats) and, when lr > 0, one Adam step.
 * FSD_ERR_BREAKDOWN (weights untouched) when the prediction is not finite,
 * as for overlapping particles. */
int fsd_learned_ratio_train_step(fsd_handle* h, const float* d_pos, float target_log_ratio, float lr, float* loss,
                                 float* predicted_log_ratio, float* host_grad);
int fsd_learned_get_poly(fsd_handle* h, float* host_c, int n);
int fsd_learned_poly_train_step(fsd_handle* h, const float* d_pos, int n_probes, unsigned int step, float lr,
                                int natural, float* loss, float* loss_opt, float* host_grad, float* host_coef,
                                float* host_coef_opt);
/* x = P^-1 b (Saddle_Preconditioner, Saddle.cu:171).  x and b may alias. */
int fsd_precond_apply(fsd_handle* h, const float* d_b, float* d_x);
/* Preconditioned GMRES on the saddle system (Solvers_Saddle, Solvers.cu:55).
 * d_x holds the initial guess on entry and the solution on exit. */
int fsd_saddle_solve(fsd_handle* h, const float* d_pos, const float* d_rhs, float* d_x, int* iters, float* resid);

/* Brownian pieces (Brownian_FarField.cu:829, Brownian_NearField.cu:407,
 * Integrator.cu:549).  Outputs are velocities/forces already scaled by
 * sqrt(2 kT / dt); draws are counter-based from (seed, timestep, stream id). */
int fsd_brownian_farfield(fsd_handle* h, const float* d_pos, unsigned int timestep, float* d_slip11);
int fsd_brownian_nearfield(fsd_handle* h, const float* d_pos, unsigned int timestep, float* d_force6);
int fsd_rfd_drift(fsd_handle* h, const float* d_pos, const int* d_image, unsigned int timestep, float* d_drift6);
/* The normals behind those draws: n values of stream `stream_id` at
 * `timestep`, times `scale`, from the counter-based Philox4x32-10 generator
 * keyed by the handle's hashed seed.  Streams: 1 far-field real-space (11N),
 * 2 wave-space field, 3 near-field (6N), 4 drift direction psi (6N),
 * 5 rotational noise (3N), 6 start vectors of spectral estimates, 7 probe
 * vectors of the learned preconditioner's training.  The reference draws
 * the first five with cuRAND
 * (Integrator.cu:591-596, Brownian_FarField.cu:864-874,
 * Brownian_NearField.cu:438-444), so this has no counterpart there; it lets a
 * caller reproduce the noise of any step. */
int fsd_draw_normals(fsd_handle* h, unsigned int stream_id, unsigned int timestep, size_t n, float scale,
                     float* d_out);
/* Explicit Euler update with simple shear, director rotation, image and
 * unwrapped-position bookkeeping from the velocity already in a->d_velocity
 * (Integrator_ExplicitEuler_Shear_kernel, Integrator.cu:126-228, launched at
 * Stokes.cu:248).  Rotational noise comes from a->d_noise_ang, or is drawn
 * from stream 5 when it is NULL and rot_diff > 0, as fsd_step does. */
int fsd_integrate_euler(fsd_handle* h, const fsd_step_args* a);

/* Velocities and stresslets for the current configuration without moving
 * particles (Integrator_ComputeVelocity, Integrator.cu:744). */
int fsd_compute_velocity(fsd_handle* h, const fsd_step_args* a);
/* One full time step (Stokes_StepOne, Stokes.cu:119).  FSD_ERR_GMRES_MAXIT
 * and FSD_ERR_LANCZOS_MAXIT from fsd_step and fsd_compute_velocity mean the
 * step completed with the best solution or sample reached (fsd_solve_info
 * has the residuals), as the reference prints a warning and continues
 * (Solvers.cu:121-125, Brownian_FarField.cu:787-794); other errors stop the
 * step before the particles move. */
int fsd_step(fsd_handle* h, const fsd_step_args* a);
/* One step of each of n independent suspensions (no counterpart in the
 * reference, which steps one system per process).  Handle i takes args[i];
 * the steps run concurrently on nthreads host threads (0: one per handle),
 * so handles created on distinct streams overlap their kernels on the GPU.
 * status (optional, n entries) receives each step's fsd_status; the return
 * value is the first error other than FSD_ERR_LANCZOS_MAXIT, or FSD_OK.
 * A handle must not appear twice in one batch. */
int fsd_step_batch(fsd_handle* const* hs, const fsd_step_args* args, int n, int nthreads, int* status);

#ifdef __cplusplus
}
#endif
#endif /* FSD_H */
