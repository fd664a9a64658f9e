// Near-field lubrication pair products over the neighbour list
// (Lubrication.cu of the reference).  Each particle owns its output row and
// sums over its own neighbours, so results are deterministic and no atomics
// are needed; a group of 8 lanes splits a particle's neighbours and reduces
// with shuffles.  The list is the neighbour list cut at rlub plus the list
// buffer (same order, so the same sums), and particles are visited in cell
// order so that a block's gathers overlap.  The resistance scalars are interpolated from the tabulated
// Jeffrey-Onishi functions exactly as the reference does (res_interp).
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_profile.h"

namespace fsd {

constexpr int kLubGroup = 8;

struct LubArgs {
    const float4* pos;
    const unsigned* order;  // particles in cell order
    const unsigned* nneigh;
    const unsigned* nlist;
    int stride;
    ResTable tab;
    Box box;
    int N;
    float rlub2;
};

// Imposed + active rate of strain of one particle as a symmetric 3x3
// (Lubrication.cu:380-410): E = (xx-zz, 2xy, 2xz, 2yz, yy-zz) -> tensor.
__device__ __forceinline__ void strain_block(float shear_rate, const float3* ori, const float* b2mask, float B2, int i,
                                             float E[3][3]) {
    float e[5] = {0.0f, shear_rate, 0.0f, 0.0f, 0.0f};
    if (B2 != 0.0f && ori) {
        const float3 p = ori[i];
        const float b2 = 0.6f * B2 * (b2mask ? b2mask[i] : 1.0f);
        e[0] += b2 * (p.x * p.x - p.z * p.z);
        e[1] += b2 * (2.f * p.x * p.y);
        e[2] += b2 * (2.f * p.x * p.z);
        e[3] += b2 * (2.f * p.y * p.z);
        e[4] += b2 * (p.y * p.y - p.z * p.z);
    }
    E[0][0] = (1.0f / 3.0f) * (2.0f * e[0] - e[4]);
    E[0][1] = 0.5f * e[1];
    E[0][2] = 0.5f * e[2];
    E[1][0] = E[0][1];
    E[1][1] = (1.0f / 3.0f) * (-e[0] + 2.0f * e[4]);
    E[1][2] = 0.5f * e[3];
    E[2][0] = E[0][2];
    E[2][1] = E[1][2];
    E[2][2] = (-1.0f / 3.0f) * (e[0] + e[4]);
}

__device__ __forceinline__ float3 eps_dot(float3 r, float3 v) {
    return make_float3(r.z * v.y - r.y * v.z, -r.z * v.x + r.x * v.z, r.y * v.x - r.x * v.y);
}

// F = R_FU U (Lubrication_RFU_kernel, Lubrication.cu:69-309).  With saddle_x,
// writes saddle_x[6i + c] - F instead (Saddle.cu:141-148).
__global__ void __launch_bounds__(128) k_rfu(LubArgs a, const float* __restrict__ U, float* __restrict__ out,
                                             const float* __restrict__ saddle_x) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / kLubGroup;
    const int gl = threadIdx.x % kLubGroup;
    const bool valid = gid < a.N;
    const int i = (int)a.order[valid ? gid : a.N - 1];
    const float4 pi = a.pos[i];
    const float3 ui = make_float3(U[6 * i], U[6 * i + 1], U[6 * i + 2]);
    const float3 wi = make_float3(U[6 * i + 3], U[6 * i + 4], U[6 * i + 5]);
    float f[6] = {0, 0, 0, 0, 0, 0};
    const unsigned nn = valid ? a.nneigh[i] : 0u;
    const unsigned* row = a.nlist + (size_t)i * a.stride;
    for (unsigned q = gl; q < nn; q += kLubGroup) {
        const unsigned j = row[q];
        const float4 pj = a.pos[j];
        const float3 R = min_image_rn(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), a.box);
        const float d2 = dist2_rn(R);
        if (!(d2 < a.rlub2 && d2 > 0.f)) continue;
        const float dist = sqrtf(d2);
        float c[10];
        res_interp<10>(a.tab, dist, 0, c);
        const float XA11 = c[0], XA12 = c[1], YA11 = c[2], YA12 = c[3], YB11 = c[4], YB12 = c[5];
        const float XC11 = c[6], XC12 = c[7], YC11 = c[8], YC12 = c[9];
        const float3 uj = make_float3(U[6 * j], U[6 * j + 1], U[6 * j + 2]);
        const float3 wj = make_float3(U[6 * j + 3], U[6 * j + 4], U[6 * j + 5]);
        const float3 r = make_float3(R.x / dist, R.y / dist, R.z / dist);
        const float rdui = r.x * ui.x + r.y * ui.y + r.z * ui.z;
        const float rduj = r.x * uj.x + r.y * uj.y + r.z * uj.z;
        const float rdwi = r.x * wi.x + r.y * wi.y + r.z * wi.z;
        const float rdwj = r.x * wj.x + r.y * wj.y + r.z * wj.z;
        const float3 eui = eps_dot(r, ui), ewi = eps_dot(r, wi), euj = eps_dot(r, uj), ewj = eps_dot(r, wj);
        const float YB21 = -YB12;
        f[0] += (XA11 - YA11) * rdui * r.x + YA11 * ui.x + (XA12 - YA12) * rduj * r.x + YA12 * uj.x + YB11 * (-ewi.x) +
                YB21 * (-ewj.x);
        f[1] += (XA11 - YA11) * rdui * r.y + YA11 * ui.y + (XA12 - YA12) * rduj * r.y + YA12 * uj.y + YB11 * (-ewi.y) +
                YB21 * (-ewj.y);
        f[2] += (XA11 - YA11) * rdui * r.z + YA11 * ui.z + (XA12 - YA12) * rduj * r.z + YA12 * uj.z + YB11 * (-ewi.z) +
                YB21 * (-ewj.z);
        f[3] += YB11 * eui.x + YB12 * euj.x + (XC11 - YC11) * rdwi * r.x + YC11 * wi.x + (XC12 - YC12) * rdwj * r.x +
                YC12 * wj.x;
        f[4] += YB11 * eui.y + YB12 * euj.y + (XC11 - YC11) * rdwi * r.y + YC11 * wi.y + (XC12 - YC12) * rdwj * r.y +
                YC12 * wj.y;
        f[5] += YB11 * eui.z + YB12 * euj.z + (XC11 - YC11) * rdwi * r.z + YC11 * wi.z + (XC12 - YC12) * rdwj * r.z +
                YC12 * wj.z;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] = group_sum<kLubGroup>(f[c]);
    if (!valid || gl != 0) return;
    if (saddle_x) {
#pragma unroll
        for (int c = 0; c < 6; ++c) out[6 * i + c] = saddle_x[6 * i + c] - f[c];
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) out[6 * i + c] = f[c];
    }
}

// F += R_FE : E (Lubrication_RFE_kernel, Lubrication.cu:350-608).
__global__ void __launch_bounds__(128) k_rfe(LubArgs a, float shear_rate, const float3* ori, const float* b2mask,
                                             float B2, float* __restrict__ out) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / kLubGroup;
    const int gl = threadIdx.x % kLubGroup;
    const bool valid = gid < a.N;
    const int i = (int)a.order[valid ? gid : a.N - 1];
    const float4 pi = a.pos[i];
    float Ei[3][3], Ej[3][3];
    strain_block(shear_rate, ori, b2mask, B2, i, Ei);
    float f[6] = {0, 0, 0, 0, 0, 0};
    const unsigned nn = valid ? a.nneigh[i] : 0u;
    const unsigned* row = a.nlist + (size_t)i * a.stride;
    for (unsigned q = gl; q < nn; q += kLubGroup) {
        const unsigned j = row[q];
        const float4 pj = a.pos[j];
        const float3 R = min_image_rn(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), a.box);
        const float d2 = dist2_rn(R);
        if (!(d2 < a.rlub2)) continue;
        const float dist = sqrtf(d2);
        float c[6];
        res_interp<6>(a.tab, dist, 10, c);
        const float XG11 = c[0], XG12 = c[1], YG11 = c[2], YG12 = c[3], YH11 = c[4], YH12 = c[5];
        strain_block(shear_rate, ori, b2mask, B2, j, Ej);
        const float3 r = make_float3(R.x / dist, R.y / dist, R.z / dist);
        const float3 Edri = make_float3(Ei[0][0] * r.x + Ei[0][1] * r.y + Ei[0][2] * r.z,
                                        Ei[1][0] * r.x + Ei[1][1] * r.y + Ei[1][2] * r.z,
                                        Ei[2][0] * r.x + Ei[2][1] * r.y + Ei[2][2] * r.z);
        const float3 Edrj = make_float3(Ej[0][0] * r.x + Ej[0][1] * r.y + Ej[0][2] * r.z,
                                        Ej[1][0] * r.x + Ej[1][1] * r.y + Ej[1][2] * r.z,
                                        Ej[2][0] * r.x + Ej[2][1] * r.y + Ej[2][2] * r.z);
        const float rdEdri = r.x * Edri.x + r.y * Edri.y + r.z * Edri.z;
        const float rdEdrj = r.x * Edrj.x + r.y * Edrj.y + r.z * Edrj.z;
        const float3 ei = eps_dot(r, Edri), ej = eps_dot(r, Edrj);
        const float XG21 = -XG12, YG21 = -YG12, YH21 = YH12;
        f[0] += (XG11 - 2.0f * YG11) * (-rdEdri) * r.x + 2.0f * YG11 * (-Edri.x) + (XG21 - 2.0f * YG21) * (-rdEdrj) * r.x +
                2.0f * YG21 * (-Edrj.x);
        f[1] += (XG11 - 2.0f * YG11) * (-rdEdri) * r.y + 2.0f * YG11 * (-Edri.y) + (XG21 - 2.0f * YG21) * (-rdEdrj) * r.y +
                2.0f * YG21 * (-Edrj.y);
        f[2] += (XG11 - 2.0f * YG11) * (-rdEdri) * r.z + 2.0f * YG11 * (-Edri.z) + (XG21 - 2.0f * YG21) * (-rdEdrj) * r.z +
                2.0f * YG21 * (-Edrj.z);
        f[3] += YH11 * (2.0f * ei.x) + YH21 * (2.0f * ej.x);
        f[4] += YH11 * (2.0f * ei.y) + YH21 * (2.0f * ej.y);
        f[5] += YH11 * (2.0f * ei.z) + YH21 * (2.0f * ej.z);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] = group_sum<kLubGroup>(f[c]);
    if (!valid || gl != 0) return;
#pragma unroll
    for (int c = 0; c < 6; ++c) out[6 * i + c] += f[c];
}

// Components (xx, xy, xz, yz, yy) of the stresslet.
__constant__ int kSa[5] = {0, 0, 0, 1, 1};
__constant__ int kSb[5] = {0, 1, 2, 2, 1};

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// S -= R_SU U (Lubrication_RSU_kernel, Lubrication.cu:650-911).
__global__ void __launch_bounds__(128) k_rsu(LubArgs a, const float* __restrict__ U, float* __restrict__ S) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / kLubGroup;
    const int gl = threadIdx.x % kLubGroup;
    const bool valid = gid < a.N;
    const int i = (int)a.order[valid ? gid : a.N - 1];
    const float4 pi = a.pos[i];
    const float3 ui = make_float3(U[6 * i], U[6 * i + 1], U[6 * i + 2]);
    const float3 wi = make_float3(U[6 * i + 3], U[6 * i + 4], U[6 * i + 5]);
    float s[5] = {0, 0, 0, 0, 0};
    const unsigned nn = valid ? a.nneigh[i] : 0u;
    const unsigned* row = a.nlist + (size_t)i * a.stride;
    for (unsigned q = gl; q < nn; q += kLubGroup) {
        const unsigned j = row[q];
        const float4 pj = a.pos[j];
        const float3 R = min_image_rn(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), a.box);
        const float d2 = dist2_rn(R);
        if (!(d2 < a.rlub2)) continue;
        const float dist = sqrtf(d2);
        float c[6];
        res_interp<6>(a.tab, dist, 10, c);
        const float XG11 = c[0], XG12 = c[1], YG11 = c[2], YG12 = c[3], YH11 = c[4], YH12 = c[5];
        const float3 uj = make_float3(U[6 * j], U[6 * j + 1], U[6 * j + 2]);
        const float3 wj = make_float3(U[6 * j + 3], U[6 * j + 4], U[6 * j + 5]);
        const float3 r = make_float3(R.x / dist, R.y / dist, R.z / dist);
        const float rdui = r.x * ui.x + r.y * ui.y + r.z * ui.z;
        const float rduj = r.x * uj.x + r.y * uj.y + r.z * uj.z;
        const float3 ewi = eps_dot(r, wi), ewj = eps_dot(r, wj);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int A = kSa[k], B = kSb[k];
            const float ra = comp(r, A), rb = comp(r, B);
            const float P = ra * rb - (A == B ? 1.0f / 3.0f : 0.0f);
            s[k] += XG11 * P * rdui + XG12 * P * rduj + YG11 * (comp(ui, A) * rb + ra * comp(ui, B) - 2.0f * ra * rb * rdui) +
                    YG12 * (comp(uj, A) * rb + ra * comp(uj, B) - 2.0f * ra * rb * rduj);
            s[k] += YH11 * (ra * comp(ewi, B) + comp(ewi, A) * rb) + YH12 * (ra * comp(ewj, B) + comp(ewj, A) * rb);
        }
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) s[c] = group_sum<kLubGroup>(s[c]);
    if (!valid || gl != 0) return;
#pragma unroll
    for (int c = 0; c < 5; ++c) S[5 * i + c] -= s[c];
}

// S += R_SE : E (Lubrication_RSE_kernel, Lubrication.cu:953-1230); pairs
// within r^2 < 16 as the reference hard-codes.
__global__ void __launch_bounds__(128) k_rse(LubArgs a, float shear_rate, const float3* ori, const float* b2mask,
                                             float B2, float* __restrict__ S) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / kLubGroup;
    const int gl = threadIdx.x % kLubGroup;
    const bool valid = gid < a.N;
    const int i = (int)a.order[valid ? gid : a.N - 1];
    const float4 pi = a.pos[i];
    float Ei[3][3], Ej[3][3];
    strain_block(shear_rate, ori, b2mask, B2, i, Ei);
    float s[5] = {0, 0, 0, 0, 0};
    const unsigned nn = valid ? a.nneigh[i] : 0u;
    const unsigned* row = a.nlist + (size_t)i * a.stride;
    for (unsigned q = gl; q < nn; q += kLubGroup) {
        const unsigned j = row[q];
        const float4 pj = a.pos[j];
        const float3 R = min_image_rn(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), a.box);
        const float d2 = dist2_rn(R);
        if (!(d2 < 16.0f)) continue;
        const float dist = sqrtf(d2);
        float c[6];
        res_interp<6>(a.tab, dist, 16, c);
        const float XM11 = c[0], XM12 = c[1], YM11 = c[2], YM12 = c[3], ZM11 = c[4], ZM12 = c[5];
        strain_block(shear_rate, ori, b2mask, B2, j, Ej);
        const float3 r = make_float3(R.x / dist, R.y / dist, R.z / dist);
        const float3 Edri = make_float3(Ei[0][0] * r.x + Ei[0][1] * r.y + Ei[0][2] * r.z,
                                        Ei[1][0] * r.x + Ei[1][1] * r.y + Ei[1][2] * r.z,
                                        Ei[2][0] * r.x + Ei[2][1] * r.y + Ei[2][2] * r.z);
        const float3 Edrj = make_float3(Ej[0][0] * r.x + Ej[0][1] * r.y + Ej[0][2] * r.z,
                                        Ej[1][0] * r.x + Ej[1][1] * r.y + Ej[1][2] * r.z,
                                        Ej[2][0] * r.x + Ej[2][1] * r.y + Ej[2][2] * r.z);
        const float rdEdri = r.x * Edri.x + r.y * Edri.y + r.z * Edri.z;
        const float rdEdrj = r.x * Edrj.x + r.y * Edrj.y + r.z * Edrj.z;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int A = kSa[k], B = kSb[k];
            const float ra = comp(r, A), rb = comp(r, B);
            const float dab = (A == B) ? 1.0f : 0.0f;
            const float P = ra * rb - dab / 3.0f;
            s[k] += 1.5f * XM11 * P * rdEdri + 1.5f * XM12 * P * rdEdrj +
                    0.5f * YM11 * (2.0f * ra * comp(Edri, B) + 2.0f * rb * comp(Edri, A) - 4.0f * rdEdri * ra * rb) +
                    0.5f * YM12 * (2.0f * ra * comp(Edrj, B) + 2.0f * rb * comp(Edrj, A) - 4.0f * rdEdrj * ra * rb) +
                    0.5f * ZM11 *
                        (2.0f * Ei[A][B] + (dab + ra * rb) * rdEdri - 2.0f * ra * comp(Edri, B) - 2.0f * rb * comp(Edri, A)) +
                    0.5f * ZM12 *
                        (2.0f * Ej[A][B] + (dab + ra * rb) * rdEdrj - 2.0f * ra * comp(Edrj, B) - 2.0f * rb * comp(Edrj, A));
        }
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) s[c] = group_sum<kLubGroup>(s[c]);
    if (!valid || gl != 0) return;
#pragma unroll
    for (int c = 0; c < 5; ++c) S[5 * i + c] += s[c];
}

static LubArgs lub_args(fsd_handle* h, const float4* pos) {
    LubArgs a;
    a.pos = pos;
    a.order = h->w.order;
    a.nneigh = h->w.lub_n;
    a.nlist = h->w.lub_list;
    a.stride = h->w.nl_stride;
    a.tab.dist = h->d_res_dist;
    a.tab.vals = h->d_res_vals;
    a.box = h->box;
    a.N = h->p.N;
    a.rlub2 = h->p.rlub * h->p.rlub;
    return a;
}

static int lub_blocks(int N) { return (N * kLubGroup + 127) / 128; }

void lub_rfu(fsd_handle* h, const float4* pos, const float* U, float* F, const float* saddle_x) {
    ProfRegion pr(h, R_RFU);
    count_launch();
    k_rfu<<<lub_blocks(h->p.N), 128, 0, h->stream>>>(lub_args(h, pos), U, F, saddle_x);
}
void lub_rfe(fsd_handle* h, const float4* pos, float shear_rate, const float3* ori, const float* b2mask, float B2,
             float* F) {
    ProfRegion pr(h, R_LUB_OTHER);
    count_launch();
    k_rfe<<<lub_blocks(h->p.N), 128, 0, h->stream>>>(lub_args(h, pos), shear_rate, ori, b2mask, B2, F);
}
void lub_rsu(fsd_handle* h, const float4* pos, const float* U, float* S) {
    ProfRegion pr(h, R_LUB_OTHER);
    count_launch();
    k_rsu<<<lub_blocks(h->p.N), 128, 0, h->stream>>>(lub_args(h, pos), U, S);
}
void lub_rse(fsd_handle* h, const float4* pos, float shear_rate, const float3* ori, const float* b2mask, float B2,
             float* S) {
    ProfRegion pr(h, R_LUB_OTHER);
    count_launch();
    k_rse<<<lub_blocks(h->p.N), 128, 0, h->stream>>>(lub_args(h, pos), shear_rate, ori, b2mask, B2, S);
}

}  // namespace fsd
