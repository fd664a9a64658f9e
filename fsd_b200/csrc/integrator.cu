// One FSD time step (Stokes_StepOne, Stokes.cu:119-273, and
// Integrator_ComputeVelocity, Integrator.cu:744-938):
//   neighbour list -> preconditioner -> pair forces -> Brownian pieces ->
//   right-hand side -> saddle solve -> stresslet (output steps) -> Euler with
//   simple shear.
#include <cmath>

#include "fsd_brownian.h"
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_profile.h"
#include "fsd_solver.h"

namespace fsd {

// Electrostatic repulsion, van der Waals attraction and stiff collisions over
// the neighbour list, plus the external torque about z
// (Stokes_SetForce_manually_kernel, Helper_Stokes.cu:65-172).
__global__ void k_pair_force(const float4* __restrict__ pos, int N, Box b, const unsigned* __restrict__ nneigh,
                             const unsigned* __restrict__ nlist, int stride, float ndsr, float k_n, float kappa,
                             float beta, float epsq, float T_ext, float* __restrict__ F) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 pi = pos[i];
    const float h_rough = sqrtf(epsq);
    const float rcol = 2.0f + 1.0f * h_rough;
    const float F0 = 1.0f / ndsr;
    const float Hamaker = F0 * beta;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    const unsigned nn = nneigh[i];
    for (unsigned q = 0; q < nn; ++q) {
        const unsigned j = nlist[(size_t)i * stride + q];
        const float4 pj = pos[j];
        const float3 R = min_image_rn(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), b);
        const float dist = sqrtf(dist2_rn(R));
        const float gap = dist - rcol;
        float mag = 0.f;
        if (gap >= 0.f && dist <= 2.0f + 10.0f / kappa) mag = Hamaker / (12.f * (gap * gap + epsq)) - F0 * expf(-kappa * gap);
        if (gap < 0.f) mag = Hamaker / (12.f * epsq) - F0 - k_n * fabsf(gap);
        fx += mag * R.x / dist;
        fy += mag * R.y / dist;
        fz += mag * R.z / dist;
    }
    F[6 * i] = fx;
    F[6 * i + 1] = fy;
    F[6 * i + 2] = fz;
    F[6 * i + 3] = 0.f;
    F[6 * i + 4] = 0.f;
    F[6 * i + 5] = T_ext;
}

// rhs[6N+5i+1] += shear rate minus the active strain; rhs[11N:] -= applied force
// (Integrator_AddStrainRate_kernel, Helper_Integrator.cu:114-158; Integrator.cu:867-869).
__global__ void k_rhs_terms(float* rhs, const float* __restrict__ force, int N, float shear_rate, float B2,
                            const float* b2mask, const float3* ori) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float* e = rhs + 6 * N + 5 * i;
    e[1] += shear_rate;
    if (B2 != 0.f && ori) {
        const float3 p = ori[i];
        const float b2 = -0.6f * B2 * (b2mask ? b2mask[i] : 1.0f);
        e[0] -= b2 * (p.x * p.x - p.z * p.z);
        e[1] -= b2 * (2.f * p.x * p.y);
        e[2] -= b2 * (2.f * p.x * p.z);
        e[3] -= b2 * (2.f * p.y * p.z);
        e[4] -= b2 * (p.y * p.y - p.z * p.z);
    }
    float* f = rhs + 11 * N + 6 * i;
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] -= force[6 * i + c];
}

__global__ void k_add(float* y, const float* x, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        y[k] += x[k];
}

// Explicit Euler with simple shear, director rotation and unwrapped
// positions (Integrator_ExplicitEuler_Shear_kernel, Integrator.cu:126-228).
__global__ void k_euler_shear(float4* pos, float3* ori, float4* pos_gb, const float* __restrict__ vel, float B1,
                              const float* b1mask, const float3* noise, int3* image, int N, Box b, float dt,
                              float shear_rate) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 p4 = pos[i];
    float3 p = make_float3(p4.x, p4.y, p4.z);
    float3 v = make_float3(vel[6 * i], vel[6 * i + 1], vel[6 * i + 2]);
    float3 w = make_float3(vel[6 * i + 3], vel[6 * i + 4], vel[6 * i + 5]);
    v.x += shear_rate * p.y;
    w.z -= shear_rate / 2.f;
    if (noise) {
        const float3 n = noise[i];
        w.x += n.x;
        w.y += n.y;
        w.z += n.z;
    }
    float q0 = 1.0f;
    float3 qv = make_float3(0.f, 0.f, 0.f);
    const float aw = sqrtf(w.x * w.x + w.y * w.y + w.z * w.z);
    if (aw > 1e-6f) {
        const float ang = aw * dt;
        q0 = cosf(ang / 2.f);
        const float s = sinf(ang / 2.f) / aw;
        qv = make_float3(w.x * s, w.y * s, w.z * s);
    }
    float3 pv = ori ? ori[i] : make_float3(0.f, 0.f, 1.f);
    const float ab = -2.f / 3.f * B1 * (b1mask ? b1mask[i] : 1.0f);
    v.x -= ab * pv.x;
    v.y -= ab * pv.y;
    v.z -= ab * pv.z;
    if (pos_gb) {
        float4 g = pos_gb[i];
        g.x += (v.x - shear_rate * p.y + shear_rate * g.y) * dt;
        g.y += v.y * dt;
        g.z += v.z * dt;
        pos_gb[i] = g;
    }
    p.x += v.x * dt;
    p.y += v.y * dt;
    p.z += v.z * dt;
    int3 img = image ? image[i] : make_int3(0, 0, 0);
    wrap_position(p, img, b);
    pos[i] = make_float4(p.x, p.y, p.z, p4.w);
    if (image) image[i] = img;
    if (ori) {
        const float qq = qv.x * qv.x + qv.y * qv.y + qv.z * qv.z;
        const float qp = qv.x * pv.x + qv.y * pv.y + qv.z * pv.z;
        float3 pn = make_float3((q0 * q0 - qq) * pv.x, (q0 * q0 - qq) * pv.y, (q0 * q0 - qq) * pv.z);
        pn.x += 2.f * qp * qv.x + 2.f * q0 * (qv.y * pv.z - qv.z * pv.y);
        pn.y += 2.f * qp * qv.y + 2.f * q0 * (qv.z * pv.x - qv.x * pv.z);
        pn.z += 2.f * qp * qv.z + 2.f * q0 * (qv.x * pv.y - qv.y * pv.x);
        const float nm = sqrtf(pn.x * pn.x + pn.y * pn.y + pn.z * pn.z);
        ori[i] = make_float3(pn.x / nm, pn.y / nm, pn.z / nm);
    }
}

// Quaternion rotation of director pv about w by |w| t, renormalised.
__device__ __forceinline__ float3 rotate_director(float3 pv, float3 w, float t) {
    float q0 = 1.0f;
    float3 qv = make_float3(0.f, 0.f, 0.f);
    const float aw = sqrtf(w.x * w.x + w.y * w.y + w.z * w.z);
    if (aw > 1e-6f) {
        const float ang = aw * t;
        q0 = cosf(ang / 2.f);
        const float s = sinf(ang / 2.f) / aw;
        qv = make_float3(w.x * s, w.y * s, w.z * s);
    }
    const float qq = qv.x * qv.x + qv.y * qv.y + qv.z * qv.z;
    const float qp = qv.x * pv.x + qv.y * pv.y + qv.z * pv.z;
    float3 pn = make_float3((q0 * q0 - qq) * pv.x, (q0 * q0 - qq) * pv.y, (q0 * q0 - qq) * pv.z);
    pn.x += 2.f * qp * qv.x + 2.f * q0 * (qv.y * pv.z - qv.z * pv.y);
    pn.y += 2.f * qp * qv.y + 2.f * q0 * (qv.z * pv.x - qv.x * pv.z);
    pn.z += 2.f * qp * qv.z + 2.f * q0 * (qv.x * pv.y - qv.y * pv.x);
    const float nm = sqrtf(pn.x * pn.x + pn.y * pn.y + pn.z * pn.z);
    return make_float3(pn.x / nm, pn.y / nm, pn.z / nm);
}

// Stage 1 of the two-stage Runge-Kutta step (Integrator_ExplicitEuler1_Shear_kernel,
// Integrator.cu:232-330): the Euler predictor x* = x + U dt, kept unwrapped
// for the average of stage 2 (and wrapped into the box for the velocity at
// x*), the director rotated by the full step, and half a step of the
// unwrapped positions.
__global__ void k_rk_stage1(const float4* __restrict__ pos, const float3* ori, float4* __restrict__ pos_star,
                            float4* __restrict__ pos_star_w, float3* ori_star, float4* pos_gb,
                            const float* __restrict__ vel, float B1, const float* b1mask, const float3* noise, int N,
                            Box b, float dt, float shear_rate) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 p4 = pos[i];
    float3 p = make_float3(p4.x, p4.y, p4.z);
    float3 v = make_float3(vel[6 * i], vel[6 * i + 1], vel[6 * i + 2]);
    float3 w = make_float3(vel[6 * i + 3], vel[6 * i + 4], vel[6 * i + 5]);
    v.x += shear_rate * p.y;
    w.z -= shear_rate / 2.f;
    if (noise) {
        const float3 n = noise[i];
        w.x += n.x;
        w.y += n.y;
        w.z += n.z;
    }
    const float3 pv = ori ? ori[i] : make_float3(0.f, 0.f, 1.f);
    const float ab = -2.f / 3.f * B1 * (b1mask ? b1mask[i] : 1.0f);
    v.x -= ab * pv.x;
    v.y -= ab * pv.y;
    v.z -= ab * pv.z;
    if (pos_gb) {
        float4 g = pos_gb[i];
        g.x += (v.x - shear_rate * p.y + shear_rate * g.y) * 0.5f * dt;
        g.y += v.y * 0.5f * dt;
        g.z += v.z * 0.5f * dt;
        pos_gb[i] = g;
    }
    p.x += v.x * dt;
    p.y += v.y * dt;
    p.z += v.z * dt;
    pos_star[i] = make_float4(p.x, p.y, p.z, p4.w);
    int3 img = make_int3(0, 0, 0);
    wrap_position(p, img, b);
    pos_star_w[i] = make_float4(p.x, p.y, p.z, p4.w);
    if (ori) ori_star[i] = rotate_director(pv, w, dt);
}

// Stage 2 (Integrator_RK_Shear_kernel, Integrator.cu:333-438): from the
// combination c1 x + c2 x* (directors likewise, renormalised) move by
// c3 dt with the velocity at the predictor, rotate by c3 dt, add half a step
// to the unwrapped positions and wrap.
__global__ void k_rk_stage2(float4* pos, float3* ori, const float4* __restrict__ pos_star,
                            const float3* __restrict__ ori_star, float4* pos_gb, const float* __restrict__ vel,
                            float B1, const float* b1mask, const float3* noise, int3* image, int N, Box b, float dt,
                            float shear_rate, float c1, float c2, float c3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 p1 = pos[i], p2 = pos_star[i];
    float3 p = make_float3(c1 * p1.x + c2 * p2.x, c1 * p1.y + c2 * p2.y, c1 * p1.z + c2 * p2.z);
    float3 v = make_float3(vel[6 * i], vel[6 * i + 1], vel[6 * i + 2]);
    float3 w = make_float3(vel[6 * i + 3], vel[6 * i + 4], vel[6 * i + 5]);
    v.x += shear_rate * p.y;
    w.z -= shear_rate / 2.f;
    if (noise) {
        const float3 n = noise[i];
        w.x += n.x;
        w.y += n.y;
        w.z += n.z;
    }
    float3 pv = make_float3(0.f, 0.f, 1.f);
    if (ori) {
        const float3 a = ori[i], c = ori_star[i];
        pv = make_float3(a.x * c1 + c.x * c2, a.y * c1 + c.y * c2, a.z * c1 + c.z * c2);
        const float m0 = sqrtf(pv.x * pv.x + pv.y * pv.y + pv.z * pv.z);
        pv = make_float3(pv.x / m0, pv.y / m0, pv.z / m0);
    }
    const float ab = -2.f / 3.f * B1 * (b1mask ? b1mask[i] : 1.0f);
    v.x -= ab * pv.x;
    v.y -= ab * pv.y;
    v.z -= ab * pv.z;
    if (pos_gb) {
        float4 g = pos_gb[i];
        g.x += (v.x - shear_rate * p.y + shear_rate * g.y) * 0.5f * dt;
        g.y += v.y * 0.5f * dt;
        g.z += v.z * 0.5f * dt;
        pos_gb[i] = g;
    }
    p.x += v.x * dt * c3;
    p.y += v.y * dt * c3;
    p.z += v.z * dt * c3;
    int3 img = image[i];
    wrap_position(p, img, b);
    pos[i] = make_float4(p.x, p.y, p.z, p1.w);
    image[i] = img;
    if (ori) ori[i] = rotate_director(pv, w, dt * c3);
}

// out = (a + b) / 2 on n entries (the step's reported velocity with two stages).
__global__ void k_mean2(float* out, const float* __restrict__ a, const float* __restrict__ b, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        out[k] = 0.5f * (a[k] + b[k]);
}

static int vb(size_t n) { return (int)std::min<size_t>(4 * 148, (n + 255) / 256); }

// Integrator_ComputeVelocity: velocity (11N) for the current positions.
int compute_velocity(fsd_handle* h, const fsd_step_args* a) {
    Workspace& w = h->w;
    const int N = h->p.N;
    const float4* pos = (const float4*)a->d_pos;
    cudaStream_t st = h->stream;
    const size_t n17 = 17 * (size_t)N;
    float* rhs = w.rhs;
    float* vel = a->d_velocity;
    FSD_CHECK_CUDA(cudaMemsetAsync(vel, 0, sizeof(float) * 11 * N, st));
    FSD_CHECK_CUDA(cudaMemsetAsync(rhs, 0, sizeof(float) * n17, st));
    // Neighbour list and preconditioner for these positions.
    int e = fsd_build_neighbor_list(h, a->d_pos);
    if (e != FSD_OK) return e;
    e = precond_build(h, pos);
    if (e != FSD_OK) return e;
    if (h->p.force_mode == FSD_FORCE_INTERPARTICLE) {
        ProfRegion pr(h, R_INTEGRATE);
        count_launch();
        k_pair_force<<<(N + 127) / 128, 128, 0, st>>>(pos, N, h->box, w.nneigh, w.nlist, w.nl_stride, h->p.ndsr,
                                                      h->p.k_n, h->p.kappa, h->p.beta_AF, h->p.epsq,
                                                      h->p.T_ext * cosf(h->p.omega_ext * a->timestep * h->p.dt),
                                                      a->d_force);
    }
    const uint32_t step = a->timestep;
    int lanczos_status = FSD_OK;
    int solve_status = FSD_OK;  // a solve that stopped above its tolerance (kept, reported)
    if (h->p.T > 0.f) {
        e = brownian_farfield(h, pos, step, rhs);
        if (e == FSD_ERR_LANCZOS_MAXIT) lanczos_status = e;
        else if (e != FSD_OK) return e;
        e = brownian_nearfield(h, pos, step, rhs + 11 * N);
        if (e == FSD_ERR_LANCZOS_MAXIT) lanczos_status = e;
        else if (e != FSD_OK) return e;
        e = rfd_drift(h, pos, step, vel);
        if (e == FSD_ERR_GMRES_MAXIT) solve_status = e;
        else if (e != FSD_OK) return e;
    }
    count_launch();
    k_rhs_terms<<<(N + 127) / 128, 128, 0, st>>>(rhs, a->d_force, N, a->shear_rate, h->p.sqm_B2, a->d_b2_mask,
                                                 (const float3*)a->d_ori);
    lub_rfe(h, pos, a->shear_rate, (const float3*)a->d_ori, a->d_b2_mask, h->p.sqm_B2, rhs + 11 * N);
    int it = 0;
    float res = 0.f;
    e = saddle_solve(h, pos, rhs, w.sol, h->p.solver_tol, &it, &res);
    h->info.gmres_iters[2] = it;
    h->info.gmres_resid[2] = res;
    if (e == FSD_ERR_GMRES_MAXIT) solve_status = e;
    else if (e != FSD_OK) return e;
    count_launch();
    k_add<<<vb(6 * N), 256, 0, st>>>(vel, w.sol + 11 * N, 6 * (size_t)N);
    if (h->p.period > 0 && ((int)(a->timestep + 1) % h->p.period) == 0) {
        count_launch();
        k_add<<<vb(5 * N), 256, 0, st>>>(vel + 6 * N, w.sol + 6 * N, 5 * (size_t)N);
        lub_rsu(h, pos, vel, vel + 6 * N);
        lub_rse(h, pos, a->shear_rate, (const float3*)a->d_ori, a->d_b2_mask, h->p.sqm_B2, vel + 6 * N);
    }
    FSD_CHECK_CUDA(cudaGetLastError());
    return solve_status != FSD_OK ? solve_status : lanczos_status;
}

// Outcomes after which a step still moves the particles: the solver and
// Lanczos limits, reported to the caller (the reference prints a warning and
// continues, Solvers.cu:121-125, Brownian_FarField.cu:787-794).
static bool step_continues(int e) { return e == FSD_OK || e == FSD_ERR_LANCZOS_MAXIT || e == FSD_ERR_GMRES_MAXIT; }

// Euler + shear from the velocity in a->d_velocity (Integrator.cu:126-228).
int integrate_euler(fsd_handle* h, const fsd_step_args* a) {
    const int N = h->p.N;
    ProfRegion pr(h, R_INTEGRATE);
    const float3* noise = (const float3*)a->d_noise_ang;
    if (!noise && h->p.rot_diff > 0.f) {
        gaussian(h, h->w.pc_t, 3 * (size_t)N, a->timestep, kStreamRot, sqrtf(2.0f * h->p.rot_diff / h->p.dt));
        noise = (const float3*)h->w.pc_t;
    }
    count_launch();
    k_euler_shear<<<(N + 127) / 128, 128, 0, h->stream>>>((float4*)a->d_pos, (float3*)a->d_ori, (float4*)a->d_pos_gb,
                                                           a->d_velocity, h->p.sqm_B1, a->d_b1_mask, noise,
                                                           (int3*)a->d_image, N, h->box, h->p.dt, a->shear_rate);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Two-stage Runge-Kutta (Heun) step of Integrator.cu:232-438: velocity at
// x, Euler predictor x*, velocity at x* with the same step's random draws,
// then the average of x and x* moved by half a step at the velocity of x*.
// The reported velocity is the mean of the two stages'; stresslets (on
// output steps) are those of the first stage.
static int step_rk2(fsd_handle* h, const fsd_step_args* a) {
    Workspace& w = h->w;
    const int N = h->p.N;
    cudaStream_t st = h->stream;
    int e = compute_velocity(h, a);
    if (!step_continues(e)) return e;
    int status = e;
    const float3* noise = (const float3*)a->d_noise_ang;
    if (!noise && h->p.rot_diff > 0.f) {
        gaussian(h, w.rk_noise, 3 * (size_t)N, a->timestep, kStreamRot, sqrtf(2.0f * h->p.rot_diff / h->p.dt));
        noise = (const float3*)w.rk_noise;
    }
    FSD_CHECK_CUDA(cudaMemcpyAsync(w.rk_u1, a->d_velocity, sizeof(float) * 6 * N, cudaMemcpyDeviceToDevice, st));
    {
        ProfRegion pr(h, R_INTEGRATE);
        count_launch();
        k_rk_stage1<<<(N + 127) / 128, 128, 0, st>>>((const float4*)a->d_pos, (const float3*)a->d_ori, w.rk_pos,
                                                      w.rk_posw, (float3*)w.rk_ori, (float4*)a->d_pos_gb,
                                                      a->d_velocity, h->p.sqm_B1, a->d_b1_mask, noise, N, h->box,
                                                      h->p.dt, a->shear_rate);
        FSD_CHECK_CUDA(cudaGetLastError());
    }
    fsd_step_args a2 = *a;
    a2.d_pos = (float*)w.rk_posw;
    a2.d_ori = a->d_ori ? w.rk_ori : nullptr;
    a2.d_pos_gb = nullptr;
    a2.d_velocity = w.rk_vel;
    e = compute_velocity(h, &a2);
    if (!step_continues(e)) return e;
    if (e == FSD_ERR_GMRES_MAXIT || status == FSD_OK) status = e;
    ProfRegion pr(h, R_INTEGRATE);
    count_launch();
    k_rk_stage2<<<(N + 127) / 128, 128, 0, st>>>((float4*)a->d_pos, (float3*)a->d_ori, w.rk_pos,
                                                  (const float3*)w.rk_ori, (float4*)a->d_pos_gb, w.rk_vel,
                                                  h->p.sqm_B1, a->d_b1_mask, noise, (int3*)a->d_image, N, h->box,
                                                  h->p.dt, a->shear_rate, 0.5f, 0.5f, 0.5f);
    count_launch();
    k_mean2<<<vb(6 * N), 256, 0, st>>>(a->d_velocity, w.rk_u1, w.rk_vel, 6 * (size_t)N);
    FSD_CHECK_CUDA(cudaGetLastError());
    return status;
}

int step(fsd_handle* h, const fsd_step_args* a) {
    int e;
    if (h->p.integrator == 1) {
        e = step_rk2(h, a);
        if (!step_continues(e)) return e;
    } else {
        e = compute_velocity(h, a);
        if (!step_continues(e)) return e;
        const int ee = integrate_euler(h, a);
        if (ee != FSD_OK) return ee;
    }
    // Carried solver state (Stokes.cc:1658-1666).
    const unsigned t = a->timestep;
    if (t % 100 == 0 || h->m_lanczos_ff > 50) h->m_lanczos_ff = 3;
    if (t % 100 == 0 || h->m_lanczos_nf > 50) h->m_lanczos_nf = 3;
    if (t % 5 == 0 || h->ichol_relaxer > 1024.0f) h->ichol_relaxer = 1.0f;
    h->nlist_valid = false;
    return e;
}

}  // namespace fsd

using namespace fsd;

extern "C" {

int fsd_brownian_farfield(fsd_handle* h, const float* d_pos, unsigned int timestep, float* d_slip11) {
    if (!h || !h->nlist_valid || !d_pos || !d_slip11) return FSD_ERR_BAD_PARAMS;
    return brownian_farfield(h, (const float4*)d_pos, timestep, d_slip11);
}

int fsd_brownian_nearfield(fsd_handle* h, const float* d_pos, unsigned int timestep, float* d_force6) {
    if (!h || !h->nlist_valid || !d_pos || !d_force6) return FSD_ERR_BAD_PARAMS;
    return brownian_nearfield(h, (const float4*)d_pos, timestep, d_force6);
}

int fsd_rfd_drift(fsd_handle* h, const float* d_pos, const int* d_image, unsigned int timestep, float* d_drift6) {
    (void)d_image;
    if (!h || !h->nlist_valid || !h->pc_valid || !d_pos || !d_drift6) return FSD_ERR_BAD_PARAMS;
    return rfd_drift(h, (const float4*)d_pos, timestep, d_drift6);
}

int fsd_draw_normals(fsd_handle* h, unsigned int stream_id, unsigned int timestep, size_t n, float scale,
                     float* d_out) {
    if (!h || !d_out || stream_id < 1 || stream_id > kStreamLearned) return FSD_ERR_BAD_PARAMS;
    if (n == 0) return FSD_OK;
    gaussian(h, d_out, n, timestep, stream_id, scale);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

int fsd_integrate_euler(fsd_handle* h, const fsd_step_args* a) {
    if (!h || !a || !a->d_pos || !a->d_velocity || !a->d_image) return FSD_ERR_BAD_PARAMS;
    h->nlist_valid = false;  // the particles move
    return integrate_euler(h, a);
}

int fsd_compute_velocity(fsd_handle* h, const fsd_step_args* a) {
    if (!h || !a || !a->d_pos || !a->d_force || !a->d_velocity) return FSD_ERR_BAD_PARAMS;
    const int st = compute_velocity(h, a);
    h->info.status = st;
    return st;
}

int fsd_step(fsd_handle* h, const fsd_step_args* a) {
    if (!h || !a || !a->d_pos || !a->d_force || !a->d_velocity) return FSD_ERR_BAD_PARAMS;
    if (h->p.integrator == 1 && !a->d_image) return FSD_ERR_BAD_PARAMS;
    const int st = step(h, a);
    h->info.status = st;
    return st;
}

}  // extern "C"
