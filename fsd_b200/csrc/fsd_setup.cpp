// One-time host set-up of the Positively Split Ewald (PSE) parameters:
// real-space cutoff, FFT grid, Gaussian support and splitting, and the
// real-space Ewald table with its self terms.
//
// Follows Stokes::setParams (Stokes.cc:118-696).  The scalar arithmetic keeps
// the reference's float/double mix so that grid sizes, P and eta come out
// bit-identical; the table is evaluated in __float128 and rounded to float,
// as the reference does.
#include "fsd_internal.h"

#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace fsd {

// Smallest 2^a 3^b 5^c in [8, 512] that is >= n (Stokes.cc:166-219), or n itself
// when none is (the caller rejects grids beyond 512).
static int smooth_size_at_least(int n) {
    std::vector<int> sizes;
    for (int p2 = 1; p2 <= 512; p2 *= 2)
        for (int p3 = 1; p2 * p3 <= 512; p3 *= 3)
            for (int p5 = 1; p2 * p3 * p5 <= 512; p5 *= 5)
                if (p2 * p3 * p5 >= 8) sizes.push_back(p2 * p3 * p5);
    std::sort(sizes.begin(), sizes.end());
    for (int s : sizes)
        if (n <= s) return s;
    return n;
}

int compute_grid_params(float xi, float error, float max_strain, float Lx, float Ly, float Lz, GridParams* g) {
    // Real-space cutoff and wave-space extent (Stokes.cc:131-134).
    g->ewald_cut = sqrtf(-logf(error)) / xi;
    const int kmax = int(2.0 * sqrtf(-logf(error)) * xi) + 1;
    const float L[3] = {Lx, Ly, Lz};
    for (int d = 0; d < 3; ++d)
        if (g->ewald_cut > L[d] / 2.0) return FSD_ERR_BAD_PARAMS;  // cutoff reaches an image (Stokes.cc:140)
    int n[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = int(kmax * L[d] / (2.0 * 3.1415926536) * 2.0) + 1;
        n[d] = smooth_size_at_least(n[d]);
    }
    if ((long long)n[0] * n[1] * n[2] > 512LL * 512LL * 512LL) return FSD_ERR_BAD_PARAMS;  // Stokes.cc:223
    g->Nx = n[0];
    g->Ny = n[1];
    g->Nz = n[2];
    // Support widened for spreading on a sheared grid (Fiore & Swan 2018),
    // then the Gaussian width m from erfc(m / sqrt(2 lambda)) <= error.
    const float gamma = max_strain;
    const float gamma2 = gamma * gamma;
    const float lambda = 1.0 + gamma2 / 2.0 + gamma * sqrtf(1.0 + gamma2 / 4.0);
    g->hx = Lx / float(n[0]);
    g->hy = Ly / float(n[1]);
    g->hz = Lz / float(n[2]);
    float m = 1.0f;
    while (erfcf(m / sqrtf(2.0 * lambda)) > error) m = m + 0.01;
    g->gauss_m = m;
    g->P = int(m * m / 3.1415926536) + 1;
    const float w = g->P * g->hx / 2.0;
    const float xisq = xi * xi;
    g->eta = (2.0 * w / m) * (2.0 * w / m) * (xisq);
    if (g->P > std::min(n[0], std::min(n[1], n[2]))) return FSD_ERR_BAD_PARAMS;  // Stokes.cc:254
    return FSD_OK;
}

// ---------------------------------------------------------------------------
// Real-space Ewald table.
//
// For each tabulated distance r the real-space part of the PSE-split
// Rotne-Prager-Yamakawa grand mobility is described by seven scalars:
//   UF: M = f_I (I - rr) + f_rr rr       (translation from force)
//   UC: g1, g2                            (translation from couplet)
//   DC: h1, h2, h3                        (velocity gradient from couplet)
// Each is a sum over three Gaussian shells centred at r, r+2a and r-2a,
//   sum_s [ exp(-(r_s xi)^2)/sqrt(pi) * A_s(r) + erfc(r_s xi) * B_s(r) ],
// plus, for overlapping spheres (r < 2a), the polynomial difference between
// the overlap-regularised and the non-overlapping RPY forms.  These are the
// closed forms of Fiore & Swan (2019) as tabulated at Stokes.cc:384-668.
// ---------------------------------------------------------------------------
typedef __float128 q;

namespace {
struct Shells {
    q E0, Ep, Em;  // exp(-r^2 x^2), exp(-(r+2a)^2 x^2), exp(-(r-2a)^2 x^2), each over sqrt(pi)
    q C0, Cp, Cm;  // erfc(r x), erfc((r+2a) x), erfc((r-2a) x)
    q Cn;          // erfc((2a-r) x) = 2 - Cm, kept separate as the closed forms use both
};

// The reference's quad-precision constants are double literals promoted to
// __float128 (Stokes.cc:357, 384); the same values are used here.
const q kPiQ = (q)3.1415926535897932384626433832795;

Shells shells(q r, q a, q x) {
    const q rs_pi = 1 / sqrtq(kPiQ);
    Shells s;
    s.E0 = expq(-(r * r) * (x * x)) * rs_pi;
    s.Ep = expq(-((r + 2 * a) * (r + 2 * a)) * (x * x)) * rs_pi;
    s.Em = expq(-((r - 2 * a) * (r - 2 * a)) * (x * x)) * rs_pi;
    s.C0 = erfcq(r * x);
    s.Cp = erfcq((r + 2 * a) * x);
    s.Cm = erfcq((r - 2 * a) * x);
    s.Cn = erfcq((2 * a - r) * x);
    return s;
}

struct Row {
    q fI, frr, g1, g2, h1, h2, h3;
};

// Functions for non-overlapping spheres (r >= 2a); also the base of the r < 2a forms.
Row far_forms(q r, q a, q x, const Shells& s) {
    const q a2 = a * a, a3 = a2 * a, a4 = a2 * a2, a5 = a4 * a, a6 = a3 * a3, a8 = a4 * a4;
    const q r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r8 = r4 * r4;
    const q x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x, x6 = x3 * x3, x7 = x6 * x, x8 = x4 * x4;
    const q rp = 2 * a + r, rm = r - 2 * a;  // shell centres
    const q ia = 1 / a, ia2 = ia * ia, ia4 = ia2 * ia2, ia6 = ia4 * ia2;
    const q ir = 1 / r, ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir;
    const q ix3 = 1 / x3, ix4 = 1 / x4, ix5 = 1 / x5, ix6 = 1 / x6, ix7 = 1 / x7, ix8 = 1 / x8;
    Row o;

    // UF, transverse part (I - rr).
    o.fI = -ia + a2 * ir3 / 2 + 3 * ir / 4 + ia2 * (9 * r / 32 - 3 * ir3 * ix4 / 128) +
           s.C0 * 3 * ia2 * ir3 * (-12 * r4 + ix4) / 128 +
           s.Cp * (128 * ia + 64 * a2 * ir3 + 96 * ir + ia2 * (36 * r - 3 * ir3 * ix4)) / 256 +
           s.Cn * (128 * ia - 64 * a2 * ir3 - 96 * ir + ia2 * (-36 * r + 3 * ir3 * ix4)) / 256 +
           s.E0 * 3 * ia2 * ir2 * ix3 * (1 + 6 * r2 * x2) / 64 +
           s.Ep * ia2 * ir3 * ix3 * (8 * r * a2 * x2 - 16 * a3 * x2 + a * (2 - 28 * r2 * x2) - 3 * (r + 6 * r3 * x2)) / 128 +
           s.Em * ia2 * ir3 * ix3 * (8 * r * a2 * x2 + 16 * a3 * x2 + a * (-2 + 28 * r2 * x2) - 3 * (r + 6 * r3 * x2)) / 128;

    // UF, longitudinal part rr.
    o.frr = -ia - a2 * ir3 + 3 * ir / 2 + 3 * ia2 * ir3 * (4 * r4 + ix4) / 64 +
            s.Cn * (64 * ia + 64 * a2 * ir3 - 96 * ir + ia2 * (-12 * r - 3 * ir3 * ix4)) / 128 +
            s.Cp * (64 * ia - 64 * a2 * ir3 + 96 * ir + ia2 * (12 * r + 3 * ir3 * ix4)) / 128 +
            s.E0 * 3 * ia2 * ir2 * ix3 * (-1 + 2 * r2 * x2) / 32 -
            s.Em * (2 * a + 3 * r) * ia2 * ir3 * ix3 * (-1 - 8 * a * r * x2 + 8 * a2 * x2 + 2 * r2 * x2) / 64 +
            s.Ep * (2 * a - 3 * r) * ia2 * ir3 * ix3 * (-1 + 8 * a * r * x2 + 8 * a2 * x2 + 2 * r2 * x2) / 64 -
            s.C0 * 3 * ia2 * ir3 * ix4 * (1 + 4 * r4 * x4) / 64;

    // UC, first function.
    {
        const q Wm = 15 + 5 * r2 * x2 * (3 + 64 * a4 * x4) + 512 * a6 * x6 - 256 * a * r5 * x6 + 100 * r6 * x6;
        const q Wp = 15 + 5 * r2 * x2 * (3 + 64 * a4 * x4) + 512 * a6 * x6 + 256 * a * r5 * x6 + 100 * r6 * x6;
        o.g1 = s.E0 * ia4 * ir3 * ix5 * (9 + 15 * r2 * x2 - 30 * r4 * x4) / 64 +
               s.Ep * ia4 * ir4 * ix5 *
                   (18 * a - 45 * r - 3 * rp * (-16 * a * r + 8 * a2 + 25 * r2) * x2 +
                    6 * rp * (-32 * r * a3 + 32 * a4 + 44 * a2 * r2 - 36 * a * r3 + 25 * r4) * x4) / 640 +
               s.Em * ia4 * ir4 * ix5 *
                   (-9 * (2 * a + 5 * r) + 3 * (2 * a - r) * (16 * a * r + 8 * a2 + 25 * r2) * x2 -
                    6 * (2 * a - r) * (32 * r * a3 + 32 * a4 + 44 * a2 * r2 + 36 * a * r3 + 25 * r4) * x4) / 640 +
               s.C0 * 3 * ia4 * ir4 * ix6 * (3 + 3 * r2 * x2 + 20 * r6 * x6) / 128 -
               s.Cm * 3 * ia4 * ir4 * ix6 * Wm / 1280 - s.Cp * 3 * ia4 * ir4 * ix6 * Wp / 1280;
    }

    // UC, second function.
    {
        const q Km = 24 * r * a2 + 16 * a3 + 14 * a * r2 + 5 * r3;
        const q Kp = -24 * r * a2 + 16 * a3 + 14 * a * r2 - 5 * r3;
        o.g2 = -s.E0 * 3 * ia4 * ir3 * ix5 * (3 - r2 * x2 + 2 * r4 * x4) / 64 +
               s.Em * ia4 * ir4 * ix5 * (18 * a + 45 * r - 3 * Km * x2 + 6 * Km * rm * rm * x4) / 640 +
               s.Ep * ia4 * ir4 * ix5 * (-18 * a + 45 * r + 3 * Kp * x2 - 6 * Kp * rp * rp * x4) / 640 +
               s.Cm * 3 * ia4 * ir4 * ix6 *
                   (15 - 15 * r2 * x2 + 4 * (128 * a6 - 80 * a4 * r2 + 16 * a * r5 - 5 * r6) * x6) / 1280 +
               s.C0 * 3 * ia4 * ir4 * ix6 * (-3 + 3 * r2 * x2 + 4 * r6 * x6) / 128 -
               s.Cp * 3 * ia4 * ir4 * ix6 *
                   (-15 + 15 * r2 * x2 + 4 * (-128 * a6 + 80 * a4 * r2 + 16 * a * r5 + 5 * r6) * x6) / 1280;
    }

    // DC, first function.
    {
        const q Qm = 96 * r * a3 + 48 * a4 + 80 * a2 * r2 + 40 * a * r3 + 5 * r4;
        const q Qp = -96 * r * a3 + 48 * a4 + 80 * a2 * r2 - 40 * a * r3 + 5 * r4;
        const q Cshell = -135 + 240 * (6 * a2 + r2) * x2 - 360 * r2 * (4 * a2 + r2) * x4;
        o.h1 = s.E0 * 3 * ia6 * ir4 * ix7 *
                   (27 - 2 * x2 * (15 * r2 + 2 * r4 * x2 - 4 * r6 * x4 + 48 * a2 * (3 - r2 * x2 + 2 * r4 * x4))) / 4096 +
               s.Em * 3 * ia6 * ir5 * ix7 *
                   (270 * a - 135 * r + 6 * (2 * a + 5 * r) * (12 * a2 + 5 * r2) * x2 -
                    4 * (144 * r * a4 + 96 * a5 + 64 * a3 * r2 - 30 * a * r4 - 5 * r5) * x4 +
                    8 * (2 * a - r) * (2 * a - r) * (2 * a - r) * Qm * x6) / 40960 +
               s.Ep * 3 * ia6 * ir5 * ix7 *
                   (-135 * rp - 6 * (2 * a - 5 * r) * (12 * a2 + 5 * r2) * x2 +
                    4 * (-144 * r * a4 + 96 * a5 + 64 * a3 * r2 - 30 * a * r4 + 5 * r5) * x4 - 8 * Qp * rp * rp * rp * x6) /
                   40960 +
               s.C0 * 3 * ia6 * ir5 * ix8 *
                   (27 + 8 * x2 * (-6 * r2 + 9 * r4 * x2 - 2 * r8 * x6 + 12 * a2 * (-3 + 3 * r2 * x2 + 4 * r6 * x6))) / 8192 +
               s.Cm * 3 * ia6 * ir5 * ix8 * (Cshell + 16 * Qm * rm * rm * rm * rm * x8) / 81920 +
               s.Cp * 3 * ia6 * ir5 * ix8 * (Cshell + 16 * Qp * rp * rp * rp * rp * x8) / 81920;
    }

    // DC, second function.
    {
        const q V = -45 + 8 * x2 * (60 * a2 - 6 * r2 + 9 * r2 * (4 * a2 + r2) * x2 +
                                    2 * (256 * a8 + 128 * a6 * r2 - 40 * a2 * r6 + 7 * r8) * x6);
        o.h2 = s.E0 * 9 * ia6 * ir4 * ix7 *
                   (-45 - 78 * r2 * x2 + 28 * r4 * x4 + 32 * a2 * x2 * (15 + 19 * r2 * x2 + 10 * r4 * x4) - 56 * r6 * x6) /
                   4096 +
               s.Ep * 9 * ia6 * ir5 * ix7 *
                   (45 * rp + 6 * (-20 * r * a2 + 8 * a3 + 46 * a * r2 + 13 * r3) * x2 -
                    4 * rp * (-32 * r * a3 + 16 * a4 + 48 * a2 * r2 - 56 * a * r3 + 7 * r4) * x4 +
                    8 * rp * (16 * a4 + 16 * a2 * r2 + 7 * r4) * rm * rm * x6) / 8192 +
               s.Em * 9 * ia6 * ir5 * ix7 *
                   (45 * rm - 6 * (20 * r * a2 + 8 * a3 + 46 * a * r2 - 13 * r3) * x2 +
                    4 * (2 * a - r) * (32 * r * a3 + 16 * a4 + 48 * a2 * r2 + 56 * a * r3 + 7 * r4) * x4 -
                    8 * (2 * a - r) * (16 * a4 + 16 * a2 * r2 + 7 * r4) * rp * rp * x6) / 8192 -
               s.Cm * 9 * ia6 * ir5 * ix8 * V / 16384 - s.Cp * 9 * ia6 * ir5 * ix8 * V / 16384 -
               s.C0 * 9 * ia6 * ir5 * ix8 *
                   (45 + 8 * x2 * (6 * r2 - 9 * r4 * x2 - 14 * r8 * x6 + 4 * a2 * (-15 - 9 * r2 * x2 + 20 * r6 * x6))) / 8192;
    }

    // DC, third function.
    {
        const q d = 2 * a - r, d3 = d * d * d;
        const q S = 4 * a2 + r2;
        const q t = 4 * a2 - r2, t3 = t * t * t;
        const q U = -45 + 8 * x2 * (60 * a2 + 6 * r2 - 3 * r2 * (12 * a2 + r2) * x2 + 2 * S * t3 * x6);
        o.h3 = s.E0 * 9 * ia6 * ir4 * ix7 *
                   (-45 + 18 * r2 * x2 - 4 * r4 * x4 + 32 * a2 * x2 * (15 + r2 * x2 - 2 * r4 * x4) + 8 * r6 * x6) / 4096 +
               s.Ep * 9 * ia6 * ir5 * ix7 *
                   (45 * rp + 6 * (2 * a - 3 * r) * rm * rm * x2 - 4 * d3 * S * x4 + 8 * d3 * S * rp * rp * x6) / 8192 +
               s.Em * 9 * ia6 * ir5 * ix7 *
                   (45 * rm - 6 * (2 * a + 3 * r) * rp * rp * x2 + 4 * S * rp * rp * rp * x4 -
                    8 * S * rm * rm * rp * rp * rp * x6) / 8192 -
               s.Cm * 9 * ia6 * ir5 * ix8 * U / 16384 - s.Cp * 9 * ia6 * ir5 * ix8 * U / 16384 +
               s.C0 * 9 * ia6 * ir5 * ix8 *
                   (-45 + 8 * x2 * (6 * r2 - 3 * r4 * x2 - 2 * r8 * x6 + 4 * a2 * (15 - 9 * r2 * x2 + 4 * r6 * x6))) / 8192;
    }
    return o;
}

// Overlapping spheres (r < 2a): the far forms plus the regularisation
// polynomials; the second DC function also changes its (r - 2a) shell.
Row overlap_forms(q r, q a, q x, const Shells& s) {
    Row o = far_forms(r, a, x, s);
    const q a2 = a * a, a3 = a2 * a, a4 = a2 * a2, a6 = a3 * a3, a8 = a4 * a4;
    const q r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r8 = r4 * r4;
    const q x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x6 = x3 * x3, x8 = x4 * x4;
    o.fI += -9 * r / (32 * a2) + 1 / a - a2 / (2 * r3) - 3 / (4 * r);
    o.frr += (2 * a + 3 * r) * (2 * a - r) * (2 * a - r) * (2 * a - r) / (16 * a2 * r3);
    o.g1 += 3 / (2 * r2) + 12 * a2 / (5 * r4) - 6 * r / (5 * a3) + 15 * r2 / (32 * a4);
    o.g2 += -3 * r / (10 * a3) - 12 * a2 / (5 * r4) + 3 / (2 * r2) + 3 * r2 / (32 * a4);
    o.h1 += 9 * r / (64 * a4) - 3 / (10 * a3) - 9 * a2 / (10 * r5) + 3 / (4 * r3) - 3 * r3 / (512 * a6);
    o.h3 += 9 * r / (64 * a4) + 9 * a2 / (2 * r5) - 9 / (4 * r3) - 9 * r3 / (512 * a6);
    // Second DC function: replace the far (r - 2a) shell by the overlap one.
    const q V = -45 + 8 * x2 * (60 * a2 - 6 * r2 + 9 * r2 * (4 * a2 + r2) * x2 +
                                2 * (256 * a8 + 128 * a6 * r2 - 40 * a2 * r6 + 7 * r8) * x6);
    const q ia6 = 1 / a6, ir3 = 1 / r3, ir5 = 1 / r5, ix6 = 1 / x6, ix8 = 1 / x8;
    o.h2 += s.Cm * 9 * ia6 * ir5 * ix8 * V / 16384;  // undo the far shell
    o.h2 += 63 * r / (64 * a4) - 3 / (2 * a3) + 9 * a2 / (2 * r5) - 3 / (4 * r3) - 33 * r3 / (512 * a6) +
            9 * ia6 * ir3 * ix6 / 128 - 27 * ir3 / (64 * a4 * x4) +
            s.Cn * 3 * ia6 * ir3 * ix6 *
                (-3 + 18 * a2 * x2 * (1 - 4 * r4 * x4) + 128 * a6 * x6 + 64 * a3 * r3 * x6 + 8 * r6 * x6) / 256 +
            s.Cm * 3 * ia6 * ir5 * ix8 *
                (135 + 8 * x2 * (-6 * (30 * a2 + r2) + 9 * (4 * a2 - 3 * r2) * r2 * x2 +
                                 2 * (-768 * a8 + 128 * a6 * r2 + 256 * a3 * r5 - 168 * a2 * r6 + 11 * r8) * x6)) /
                16384;
    return o;
}
}  // namespace

void ewald_table(float xi, float error, std::vector<float>& table, float* self_x, float* self_y, float* ewald_cut,
                 int* ewald_n, float* ewald_dr) {
    *ewald_cut = sqrtf(-logf(error)) / xi;
    *ewald_dr = 0.001f;
    *ewald_n = int(*ewald_cut / *ewald_dr - 1);  // Stokes.cc:354
    const int nR = *ewald_n + 1;

    // Self terms in single precision (Stokes.cc:361-371).
    const float pi12 = 1.77245385091f, pi = 3.1415926536f, aa = 1.0f;
    const float axi = aa * xi, axi2 = axi * axi;
    *self_x = (1. + 4. * pi12 * axi * erfcf(2. * axi) - expf(-4. * axi2)) / (4. * pi12 * axi * aa);
    *self_y = ((-3. * erfcf(2. * aa * xi) * powf(aa, -3.)) / 10. -
               (3. * powf(aa, -6.) * powf(pi, -0.5) * powf(xi, -3.)) / 80. -
               (9. * powf(aa, -4.) * powf(pi, -0.5) * powf(xi, -1.)) / 40. +
               (3. * expf(-4. * powf(aa, 2.) * powf(xi, 2.)) * powf(aa, -6.) * powf(pi, -0.5) * powf(xi, -3.) *
                (1. + 10. * powf(aa, 2.) * powf(xi, 2.))) / 80.);

    // Entries at r = (k+1) dr, two float4 per entry:
    //   {f_I, f_rr, g1/2, -g2/2}, {h1, h2, h3, 0}.
    table.assign(size_t(8) * nR, 0.0f);
    const q dr = (q)0.001, x = xi, a = 1;
    for (int k = 0; k < nR; ++k) {
        const q r = q(k) * dr + dr;
        const Shells s = shells(r, a, x);
        const Row o = (r < 2 * a) ? overlap_forms(r, a, x, s) : far_forms(r, a, x, s);
        float* e = &table[size_t(8) * k];
        e[0] = float(o.fI);
        e[1] = float(o.frr);
        e[2] = float(o.g1 / 2);
        e[3] = float(-o.g2 / 2);
        e[4] = float(o.h1);
        e[5] = float(o.h2);
        e[6] = float(o.h3);
        e[7] = 0.0f;
    }
}

}  // namespace fsd
