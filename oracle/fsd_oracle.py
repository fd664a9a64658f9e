"""FP64 NumPy restatement of the FSD velocity path -- TEST INFRASTRUCTURE ONLY.

Used by the tests as the checker for the CUDA path.  Every function names the
reference file:line it restates (paths relative to the reference's source/).
Arrays: positions (N,3) float, box L = (Lx, Ly, Lz) with xy tilt, generalized
vectors in the reference's 11N / 17N layouts.

Where the reference fixes a value in single precision that decides *which*
element is used (grid node of a stencil, table row), the same single-precision
arithmetic is reproduced; all sums are FP64.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

PI_REF = 3.1415926536          # the reference's pi literal
TWO_PI_KGRID = 2.0 * 3.1416926536  # Helper_Mobility.cu:389-391 (as written there)
RES_MIN = np.float32(0.000100)  # Stokes_ResistanceTable.cc:37
RES_DR = np.float32(0.004305)   # Stokes_ResistanceTable.cc:40
F32 = np.float32

_TABLE_BIN = Path(__file__).resolve().parents[1] / "fsd_b200" / "data" / "resistance_table.bin"

# Host threads the oracle's FFTs may use (scipy.fft workers); 1 by default.
FFT_WORKERS = 1


def _fftn(a, axes, inverse=False):
    import scipy.fft as sf
    f = sf.ifftn if inverse else sf.fftn
    return f(a, axes=axes, workers=FFT_WORKERS)


def scatter_add(out, idx, vals):
    """out[idx[k]] += vals[k] along the first axis (np.add.at semantics), by
    bincount per trailing component."""
    idx = np.asarray(idx).ravel()
    v = np.asarray(vals, np.float64)
    for c in np.ndindex(*out.shape[1:]):
        out[(slice(None),) + c] += np.bincount(idx, weights=v[(slice(None),) + c], minlength=out.shape[0])
    return out


# ---------------------------------------------------------------------- data
def resistance_table():
    """Tabulated Jeffrey-Onishi scalars: dist (1000,), vals (1000, 22) as float32."""
    b = np.fromfile(_TABLE_BIN, np.float32)
    return b[:1000].copy(), b[1000:].reshape(1000, 22).copy()


# ----------------------------------------------------------------- box maths
def xyz(pos):
    """Coordinates (N,3) of float4 or float3 positions."""
    return np.asarray(pos, np.float64)[:, :3]


def min_image(d, L, xy):
    """HOOMD BoxDim::minImage, device path (rint), z then y then x."""
    d = np.array(d, np.float64, copy=True)
    Lx, Ly, Lz = L
    img = np.rint(d[..., 2] / Lz)
    d[..., 2] -= Lz * img
    img = np.rint(d[..., 1] / Ly)
    d[..., 0] -= Ly * xy * img
    d[..., 1] -= Ly * img
    d[..., 0] -= Lx * np.rint(d[..., 0] / Lx)
    return d


def min_image32(d, L, xy):
    """min_image in single precision, as the kernels evaluate pair separations."""
    d = np.array(d, F32, copy=True)
    Lx, Ly, Lz = (F32(v) for v in L)
    xy = F32(xy)
    img = np.rint(d[..., 2] * (F32(1) / Lz))
    d[..., 2] -= Lz * img
    img = np.rint(d[..., 1] * (F32(1) / Ly))
    d[..., 0] -= Ly * xy * img
    d[..., 1] -= Ly * img
    d[..., 0] -= Lx * np.rint(d[..., 0] * (F32(1) / Lx))
    return d


def make_fraction32(pos, L, xy):
    """HOOMD BoxDim::makeFraction in single precision."""
    p = np.asarray(pos, F32)[:, :3]
    Lx, Ly, Lz = (F32(v) for v in L)
    d = p + np.array([Lx / F32(2), Ly / F32(2), Lz / F32(2)], F32)
    d[:, 0] = d[:, 0] - F32(xy) * p[:, 1]
    return d / np.array([Lx, Ly, Lz], F32)


# -------------------------------------------------------------------- set-up
def grid_params(xi, error, max_strain, L):
    """Stokes::setParams grid, support and splitting (Stokes.cc:131-251)."""
    xi, error, max_strain = F32(xi), F32(error), F32(max_strain)
    cut = F32(np.sqrt(-np.log(error, dtype=F32), dtype=F32) / xi)
    kmax = int(2.0 * float(F32(np.sqrt(-np.log(error, dtype=F32), dtype=F32))) * float(xi)) + 1
    sizes = sorted({2 ** a * 3 ** b * 5 ** c for a in range(10) for b in range(6) for c in range(4)
                    if 8 <= 2 ** a * 3 ** b * 5 ** c <= 512})
    n = []
    for Ld in L:
        m = int(kmax * float(F32(Ld)) / (2.0 * PI_REF) * 2.0) + 1
        n.append(next((s for s in sizes if m <= s), m))
    gamma = max_strain
    lam = F32(1.0 + float(gamma * gamma) / 2.0 + float(gamma) * float(np.sqrt(F32(1.0 + float(gamma * gamma) / 4.0), dtype=F32)))
    h = [F32(F32(Ld) / F32(nd)) for Ld, nd in zip(L, n)]
    from math import erfc
    m = F32(1.0)
    while F32(erfc(float(F32(m / F32(np.sqrt(F32(2.0 * float(lam)), dtype=F32)))))) > error:
        m = F32(float(m) + 0.01)
    P = int(float(m * m) / PI_REF) + 1
    w = F32(P * float(h[0]) / 2.0)
    eta = F32((2.0 * float(w) / float(m)) ** 2 * float(xi * xi))
    return dict(Nx=n[0], Ny=n[1], Nz=n[2], P=P, ewald_cut=float(cut), gauss_m=float(m), eta=float(eta),
                hx=float(h[0]), hy=float(h[1]), hz=float(h[2]))


def hash_seed(seed: int) -> int:
    """Seed hash of the Stokes constructor (Stokes.cc:74)."""
    s = (seed * 0x12345677 + 0x12345) & 0xFFFFFFFF
    s ^= s >> 16
    return (s * 0x45679) & 0xFFFFFFFF


# ------------------------------------------------------------ neighbour list
def neighbor_list(pos, L, xy, rlist):
    """All j != i with |minImage(x_i - x_j)| < rlist, each row sorted."""
    pos = xyz(pos)
    N = len(pos)
    rows = []
    r2 = rlist * rlist
    for i in range(N):
        d = min_image(pos[i] - pos, L, xy)
        dd = np.einsum("ij,ij->i", d, d)
        m = dd < r2
        m[i] = False
        rows.append(np.nonzero(m)[0].astype(np.uint32))
    return rows


def neighbor_list_kdtree(pos, L, rlist):
    """neighbor_list for an untilted box by a k-d tree (same sorted rows;
    for large N, where the all-pairs scan is slow)."""
    from scipy.spatial import cKDTree
    Lb = np.asarray(L, np.float64)
    x = np.mod(xyz(pos) + Lb / 2, Lb)
    x = np.where(x >= Lb, x - Lb, x)
    pairs = cKDTree(x, boxsize=Lb).query_pairs(rlist, output_type="ndarray")
    # query_pairs keeps d <= r; the list keeps d < r
    d = min_image(xyz(pos)[pairs[:, 0]] - xyz(pos)[pairs[:, 1]], L, 0.0)
    pairs = pairs[np.einsum("ij,ij->i", d, d) < rlist * rlist]
    i = np.concatenate([pairs[:, 0], pairs[:, 1]])
    j = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    starts = np.searchsorted(i, np.arange(len(x) + 1))
    return [j[starts[k]:starts[k + 1]].astype(np.uint32) for k in range(len(x))]


def pair_arrays(rows):
    i = np.concatenate([np.full(len(r), k, np.int64) for k, r in enumerate(rows)]) if rows else np.zeros(0, np.int64)
    j = np.concatenate([np.asarray(r, np.int64) for r in rows]) if rows else np.zeros(0, np.int64)
    return i, j


# ------------------------------------------------------------------ packing
def split_generalized(genF, N):
    """Saddle_SplitGeneralizedF + Mobility_TS2C (Helper_Saddle.cu:108, Helper_Mobility.cu:294).

    Returns F (N,3) and the couplet C (N,3,3), built from torque (sign flipped)
    and stresslet (Sxx, Sxy, Sxz, Syz, Syy)."""
    g = np.asarray(genF, np.float64)
    a = g[: 6 * N].reshape(N, 6)
    s = g[6 * N: 11 * N].reshape(N, 5)
    F = a[:, :3].copy()
    Lt = -a[:, 3:6]
    Sxx, Sxy, Sxz, Syz, Syy = s.T
    C = np.zeros((N, 3, 3))
    C[:, 0, 0] = Sxx
    C[:, 0, 1] = Sxy + 0.5 * Lt[:, 2]
    C[:, 0, 2] = Sxz - 0.5 * Lt[:, 1]
    C[:, 1, 2] = Syz + 0.5 * Lt[:, 0]
    C[:, 1, 1] = Syy
    C[:, 1, 0] = Sxy - 0.5 * Lt[:, 2]
    C[:, 2, 0] = Sxz + 0.5 * Lt[:, 1]
    C[:, 2, 1] = Syz - 0.5 * Lt[:, 0]
    C[:, 2, 2] = -(Sxx + Syy)
    return F, C


def generalized_velocity(u, D, N):
    """Mobility_D2WE + Saddle_MakeGeneralizedU (Helper_Mobility.cu:235, Helper_Saddle.cu:152).

    D (N,3,3) is the velocity-gradient-like tensor whose symmetric part gives E
    and antisymmetric part Omega: W = (D_yz - D_zy, D_zx - D_xz, D_xy - D_yx)/2."""
    W = 0.5 * np.stack([D[:, 1, 2] - D[:, 2, 1], D[:, 2, 0] - D[:, 0, 2], D[:, 0, 1] - D[:, 1, 0]], 1)
    Exx, Eyy = D[:, 0, 0], D[:, 1, 1]
    Exy = 0.5 * (D[:, 0, 1] + D[:, 1, 0])
    Exz = 0.5 * (D[:, 0, 2] + D[:, 2, 0])
    Eyz = 0.5 * (D[:, 1, 2] + D[:, 2, 1])
    out = np.zeros(11 * N)
    out[: 6 * N] = np.concatenate([u, W], 1).ravel()
    out[6 * N:] = np.stack([2 * Exx + Eyy, 2 * Exy, 2 * Exz, 2 * Eyz, 2 * Eyy + Exx], 1).ravel()
    return out


# --------------------------------------------------------------- wave space
def stencil(pos, L, xy, Nxyz, P):
    """Grid nodes of each particle's P^3 support, in the reference's order
    (Mobility.cu:213-253): returns node indices (N, P^3, 3)."""
    Nx, Ny, Nz = Nxyz
    f = make_fraction32(pos, L, xy) * np.array([Nx, Ny, Nz], F32)
    x0 = f.astype(np.int64)  # truncation, as int(float)
    odd = P % 2
    start = x0 - P // 2 + 1 - odd * ((f - x0.astype(F32)) < F32(0.5)).astype(np.int64)
    t = np.stack(np.meshgrid(np.arange(P), np.arange(P), np.arange(P), indexing="ij"), -1).reshape(-1, 3)
    idx = start[:, None, :] + t[None, :, :]
    n = np.array([Nx, Ny, Nz])
    idx = np.where(idx < 0, idx + n, np.where(idx > n - 1, idx - n, idx))
    return idx


def node_positions(idx, L, xy, h):
    """Grid node coordinates on the sheared lattice (Mobility.cu:255-260)."""
    pg = idx * np.array(h) - np.array(L) / 2.0
    pg[..., 0] = pg[..., 0] + xy * pg[..., 1]
    return pg


def gridk(Nxyz, L, xy, xi, eta, pi_typo=True):
    """Wave vectors and Green's scale (Mobility_SetGridk_kernel, Helper_Mobility.cu:351-410)."""
    Nx, Ny, Nz = Nxyz
    i = np.arange(Nx)
    j = np.arange(Ny)
    k = np.arange(Nz)
    ii = np.where(i < (Nx + 1) // 2, i, i - Nx).astype(np.float64)
    jj = np.where(j < (Ny + 1) // 2, j, j - Ny).astype(np.float64)
    kk = np.where(k < (Nz + 1) // 2, k, k - Nz).astype(np.float64)
    I, J, K = np.meshgrid(ii, jj, kk, indexing="ij")
    s = TWO_PI_KGRID if pi_typo else 2.0 * np.pi
    kx = I / L[0] * s
    ky = (J - xy * I * L[1] / L[0]) / L[1] * s
    kz = K / L[2] * s
    k2 = kx * kx + ky * ky + kz * kz
    G = Nx * Ny * Nz
    with np.errstate(divide="ignore", invalid="ignore"):
        w = 6.0 * PI_REF * (1.0 + k2 / 4.0 / xi ** 2) * np.exp(-(1 - eta) * k2 / 4.0 / xi ** 2) / k2 / G
    w[0, 0, 0] = 0.0
    return kx, ky, kz, w


def green(Fh, Ch, kx, ky, kz, w):
    """Mobility_WaveSpace_Green_kernel (Mobility.cu:315-479) on full complex spectra.

    Fh: (3, ...) force spectra; Ch: (3, 3, ...) couplet spectra.  Returns
    velocity spectra (3, ...) and velocity-gradient spectra (3, 3, ...)."""
    kv = np.stack([kx, ky, kz])
    k2 = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore", invalid="ignore"):
        k = np.sqrt(k2)
        j0 = np.sin(k) / k
        j1k = (np.sin(k) - k * np.cos(k)) / (k2 * k)
        kdF = np.einsum("a...,a...->...", kv, Fh) / k2
        Cdk = np.einsum("ab...,b...->a...", Ch, kv)
        kdCdk = np.einsum("a...,a...->...", kv, Cdk) / k2
    zero = k2 == 0
    kdF[zero] = 0
    kdCdk[zero] = 0
    Buf = np.where(zero, 0, w * j0 * j0)
    Buc = np.where(zero, 0, -w * j0 * 3.0 * j1k)
    Bdf = np.where(zero, 0, w * j0 * 3.0 * j1k)
    Bdc = np.where(zero, 0, w * 9.0 * j1k * j1k)
    U = (Fh - kv * kdF) * Buf + 1j * (Cdk - kv * kdCdk) * Buc
    kk = kv[:, None] * kv[None, :]
    D = 1j * (Fh[:, None] * kv[None, :] - kk * kdF) * Bdf + (Cdk[:, None] * kv[None, :] - kk * kdCdk) * Bdc
    return U, D


def wave_space(pos, F, C, L, xy, gp, xi, pi_typo=True):
    """Wave-space part of the grand mobility (gpu_stokes_Mwave_wrap, Mobility.cu:896-1020).

    Returns u (N,3) and the contracted velocity-gradient tensor Dw (N,3,3)
    with Dw[a,b] the contraction of grid ab."""
    N = len(pos)
    Nxyz = (gp["Nx"], gp["Ny"], gp["Nz"])
    P = gp["P"]
    eta = gp["eta"]
    h = (gp["hx"], gp["hy"], gp["hz"])
    xisq = xi * xi
    prefac = (2.0 * xisq / PI_REF / eta) * np.sqrt(2.0 * xisq / PI_REF / eta)
    expfac = 2.0 * xisq / eta
    idx = stencil(pos, L, xy, Nxyz, P)
    pg = node_positions(idx, L, xy, h)
    r = min_image(pg - xyz(pos)[:, None, :], L, xy)
    wgt = prefac * np.exp(-expfac * np.einsum("npk,npk->np", r, r))
    flat = (idx[..., 0] * Nxyz[1] + idx[..., 1]) * Nxyz[2] + idx[..., 2]
    G = Nxyz[0] * Nxyz[1] * Nxyz[2]
    grids = np.zeros((12, G))
    vals = np.concatenate([F, C.reshape(N, 9)], 1)  # X Y Z, then C row-major
    for c in range(12):
        grids[c] += np.bincount(flat.ravel(), weights=(wgt * vals[:, c:c + 1]).ravel(), minlength=G)
    spec = _fftn(grids.reshape(12, *Nxyz), (1, 2, 3))
    Fh = spec[:3]
    Ch = spec[3:].reshape(3, 3, *Nxyz)
    Ch[2, 2] = -(Ch[0, 0] + Ch[1, 1])
    kx, ky, kz, w = gridk(Nxyz, L, xy, xi, eta, pi_typo)
    Uh, Dh = green(Fh, Ch, kx, ky, kz, w)
    Ur = _fftn(Uh, (1, 2, 3), inverse=True).real * G
    Dr = _fftn(Dh, (2, 3, 4), inverse=True).real * G
    quadW = h[0] * h[1] * h[2]
    cw = quadW * wgt
    u = np.einsum("np,cnp->nc", cw, Ur.reshape(3, G)[:, flat])
    Dw = np.einsum("np,abnp->nab", cw, Dr.reshape(3, 3, G)[:, :, flat])
    return u, Dw


# --------------------------------------------------------------- real space
def real_space(pos, F, C, L, xy, rows, table, self_x, self_y, ewald_cut, ewald_n, ewald_dr=1e-3):
    """Real-space Ewald sum plus self term (Mobility_RealSpace_kernel, Mobility.cu:1046-1226).

    Returns u (N,3) and D (N,3,3) in the real-space convention (D[a,b] gets
    R_a F_b-type terms)."""
    pos = xyz(pos)
    N = len(pos)
    u = self_x * F.copy()
    D = self_y * (C - 4.0 * np.transpose(C, (0, 2, 1)))
    i, j = pair_arrays(rows)
    r = min_image(pos[i] - pos[j], L, xy)
    d2 = np.einsum("ij,ij->i", r, r)
    keep = (d2 < ewald_cut ** 2) & (d2 >= ewald_dr ** 2)
    i, j, r, d2 = i[keep], j[keep], r[keep], d2[keep]
    dist = np.sqrt(d2)
    d32 = dist.astype(F32)
    rind = np.floor(F32(ewald_n) * (d32 - F32(ewald_dr)) / (F32(ewald_cut) - F32(ewald_dr))).astype(np.int64)
    # A distance that rounds up to the cutoff in float32 gives rind = n; the
    # reference then reads one row past its table.  Clamped, as the CUDA path.
    rind = np.clip(rind, 0, ewald_n - 1)
    fac = dist / ewald_dr - rind - 1.0
    t = np.asarray(table, np.float64).reshape(-1, 8)
    lo, hi = t[rind], t[rind + 1]
    v = lo + (hi - lo) * fac[:, None]
    f1, f2 = v[:, 0], v[:, 1]
    g1, g2 = -v[:, 2], -v[:, 3]
    h1, h2, h3 = v[:, 4], v[:, 5], v[:, 6]
    R = r / dist[:, None]
    Fj, Cj = F[j], C[j]
    rF = np.einsum("pa,pa->p", R, Fj)
    CR = np.einsum("pab,pb->pa", Cj, R)
    RC = np.einsum("pa,pab->pb", R, Cj)
    RCR = np.einsum("pa,pa->p", R, CR)
    du = (f1[:, None] * Fj + ((f2 - f1) * rF)[:, None] * R + g1[:, None] * (CR - RCR[:, None] * R)
          + g2[:, None] * (RC - 4.0 * RCR[:, None] * R))
    I3 = np.eye(3)
    RR = R[:, :, None] * R[:, None, :]
    dD = (-g1[:, None, None] * (R[:, :, None] * Fj[:, None, :] - rF[:, None, None] * RR)
          - g2[:, None, None] * (rF[:, None, None] * I3 + Fj[:, :, None] * R[:, None, :] - 4.0 * rF[:, None, None] * RR))
    CT = np.transpose(Cj, (0, 2, 1))
    dD += (h1[:, None, None] * (Cj - 4.0 * CT)
           + h2[:, None, None] * (R[:, :, None] * CR[:, None, :] - RCR[:, None, None] * RR)
           + h3[:, None, None] * (RCR[:, None, None] * I3 + CR[:, :, None] * R[:, None, :] + R[:, :, None] * RC[:, None, :]
                                  + RC[:, :, None] * R[:, None, :] - 6.0 * RCR[:, None, None] * RR - CT))
    scatter_add(u, i, du)
    scatter_add(D, i, dD)
    return u, D


def mobility(pos, genF, L, xy, gp, xi, rows, table, self_x, self_y, ewald_cut, ewald_n, parts=3, pi_typo=True):
    """Generalized far-field mobility (Mobility_GeneralizedMobility, Mobility.cu:1488).

    Wave and real parts are combined as the reference does: the wave-space
    gradient is stored transposed (Mobility.cu:831-833), then both are summed
    and split into (W, E)."""
    N = len(pos)
    F, C = split_generalized(genF, N)
    u = np.zeros((N, 3))
    D = np.zeros((N, 3, 3))
    if parts & 1:
        uw, Dw = wave_space(pos, F, C, L, xy, gp, xi, pi_typo)
        u += uw
        D += np.transpose(Dw, (0, 2, 1))
    if parts & 2:
        ur, Dr = real_space(pos, F, C, L, xy, rows, table, self_x, self_y, ewald_cut, ewald_n)
        u += ur
        D += Dr
    return generalized_velocity(u, D, N)


# ---------------------------------------------------------------- lubrication
def res_interp(dist, first, count, tdist, tvals, mode="lub"):
    """Interpolated resistance scalars (Lubrication.cu:172-238; Precondition.cu:612-660).

    mode 'lub': regularised row 232 for r <= 2.001; 'precond': row 0 for
    r <= 2 + 1e-4.  Rows past the end of the table (index 999) give zero."""
    d32 = np.asarray(dist, F32)
    out = np.zeros((len(d32), count))
    if mode == "lub":
        near = d32.astype(np.float64) <= 2.001
        out[near] = tvals[232, first:first + count]
    else:
        near = d32.astype(np.float64) <= 2.0 + float(RES_MIN)
        out[near] = tvals[0, first:first + count]
    far = ~near
    s = ((d32[far].astype(np.float64) - 2.0) / float(RES_MIN)).astype(F32)
    ind = (np.log10(s) / RES_DR).astype(np.int64)
    ok = ind < 999
    fi = np.nonzero(far)[0]
    ind_ok = ind[ok]
    dl = tdist[ind_ok].astype(np.float64)
    du = tdist[ind_ok + 1].astype(np.float64)
    fac = (d32[fi[ok]].astype(np.float64) - dl) / (du - dl)
    lo = tvals[ind_ok, first:first + count].astype(np.float64)
    hi = tvals[ind_ok + 1, first:first + count].astype(np.float64)
    out[fi[ok]] = lo + (hi - lo) * fac[:, None]
    return out


def _lub_pairs(pos, L, xy, rows, cut2, positive=False):
    """Pairs from i to j within the cutoff.  Separation, squared distance and
    distance are single precision as in the kernels (Lubrication.cu:126-141):
    near contact the tabulated functions are steep in the gap, so the gap's
    float32 resolution is part of the result."""
    pos = np.asarray(pos, F32)[:, :3]
    i, j = pair_arrays(rows)
    R = min_image32(pos[j] - pos[i], L, xy)  # from i to j
    d2 = R[:, 0] * R[:, 0] + R[:, 1] * R[:, 1] + R[:, 2] * R[:, 2]
    keep = d2 < F32(cut2)
    if positive:
        keep &= d2 > 0
    i, j, R, d2 = i[keep], j[keep], R[keep], d2[keep]
    dist = np.sqrt(d2)
    r = (R / dist[:, None]).astype(np.float64)
    return i, j, r, dist


def strain_tensor(shear_rate, N, ori=None, b2mask=None, B2=0.0):
    """Imposed plus active rate of strain per particle (Lubrication.cu:380-410)."""
    e = np.zeros((N, 5))
    e[:, 1] = shear_rate
    if B2 != 0.0 and ori is not None:
        p = np.asarray(ori, np.float64)
        m = np.ones(N) if b2mask is None else np.asarray(b2mask, np.float64)
        b2 = 0.6 * B2 * m
        e[:, 0] += b2 * (p[:, 0] ** 2 - p[:, 2] ** 2)
        e[:, 1] += b2 * 2 * p[:, 0] * p[:, 1]
        e[:, 2] += b2 * 2 * p[:, 0] * p[:, 2]
        e[:, 3] += b2 * 2 * p[:, 1] * p[:, 2]
        e[:, 4] += b2 * (p[:, 1] ** 2 - p[:, 2] ** 2)
    E = np.zeros((N, 3, 3))
    E[:, 0, 0] = (2 * e[:, 0] - e[:, 4]) / 3
    E[:, 1, 1] = (-e[:, 0] + 2 * e[:, 4]) / 3
    E[:, 2, 2] = -(e[:, 0] + e[:, 4]) / 3
    E[:, 0, 1] = E[:, 1, 0] = 0.5 * e[:, 1]
    E[:, 0, 2] = E[:, 2, 0] = 0.5 * e[:, 2]
    E[:, 1, 2] = E[:, 2, 1] = 0.5 * e[:, 3]
    return E


def rfu(pos, U6, L, xy, rows, tdist, tvals, rlub=4.0):
    """F = R_FU U (Lubrication_RFU_kernel, Lubrication.cu:69-309)."""
    N = len(pos)
    U = np.asarray(U6, np.float64).reshape(N, 6)
    i, j, r, dist = _lub_pairs(pos, L, xy, rows, rlub * rlub, positive=True)
    c = res_interp(dist, 0, 10, tdist, tvals)
    XA11, XA12, YA11, YA12, YB11, YB12, XC11, XC12, YC11, YC12 = c.T
    ui, wi, uj, wj = U[i, :3], U[i, 3:], U[j, :3], U[j, 3:]
    dot = lambda a, b: np.einsum("pa,pa->p", a, b)
    F = ((XA11 - YA11) * dot(r, ui))[:, None] * r + YA11[:, None] * ui + ((XA12 - YA12) * dot(r, uj))[:, None] * r \
        + YA12[:, None] * uj - YB11[:, None] * np.cross(wi, r) + YB12[:, None] * np.cross(wj, r)
    T = YB11[:, None] * np.cross(ui, r) + YB12[:, None] * np.cross(uj, r) \
        + ((XC11 - YC11) * dot(r, wi))[:, None] * r + YC11[:, None] * wi \
        + ((XC12 - YC12) * dot(r, wj))[:, None] * r + YC12[:, None] * wj
    out = np.zeros((N, 6))
    scatter_add(out, i, np.concatenate([F, T], 1))
    return out.ravel()


def rfe(pos, shear_rate, L, xy, rows, tdist, tvals, ori=None, b2mask=None, B2=0.0, rlub=4.0):
    """R_FE : E contribution (Lubrication_RFE_kernel, Lubrication.cu:350-608)."""
    N = len(pos)
    E = strain_tensor(shear_rate, N, ori, b2mask, B2)
    i, j, r, dist = _lub_pairs(pos, L, xy, rows, rlub * rlub)
    c = res_interp(dist, 10, 6, tdist, tvals)
    XG11, XG12, YG11, YG12, YH11, YH12 = c.T
    Eri = np.einsum("pab,pb->pa", E[i], r)
    Erj = np.einsum("pab,pb->pa", E[j], r)
    rEri = np.einsum("pa,pa->p", r, Eri)
    rErj = np.einsum("pa,pa->p", r, Erj)
    XG21, YG21 = -XG12, -YG12
    F = ((XG11 - 2 * YG11) * -rEri)[:, None] * r - 2 * YG11[:, None] * Eri \
        + ((XG21 - 2 * YG21) * -rErj)[:, None] * r - 2 * YG21[:, None] * Erj
    T = 2 * YH11[:, None] * np.cross(Eri, r) + 2 * YH12[:, None] * np.cross(Erj, r)
    out = np.zeros((N, 6))
    scatter_add(out, i, np.concatenate([F, T], 1))
    return out.ravel()


_SAB = [(0, 0), (0, 1), (0, 2), (1, 2), (1, 1)]


def rsu(pos, U6, L, xy, rows, tdist, tvals, rlub=4.0):
    """-R_SU U (Lubrication_RSU_kernel, Lubrication.cu:650-911)."""
    N = len(pos)
    U = np.asarray(U6, np.float64).reshape(N, 6)
    i, j, r, dist = _lub_pairs(pos, L, xy, rows, rlub * rlub)
    c = res_interp(dist, 10, 6, tdist, tvals)
    XG11, XG12, YG11, YG12, YH11, YH12 = c.T
    ui, wi, uj, wj = U[i, :3], U[i, 3:], U[j, :3], U[j, 3:]
    rui = np.einsum("pa,pa->p", r, ui)
    ruj = np.einsum("pa,pa->p", r, uj)
    ewi, ewj = np.cross(wi, r), np.cross(wj, r)
    S = np.zeros((len(i), 5))
    for k, (a, b) in enumerate(_SAB):
        P = r[:, a] * r[:, b] - (1.0 / 3.0 if a == b else 0.0)
        S[:, k] = (XG11 * P * rui + XG12 * P * ruj
                   + YG11 * (ui[:, a] * r[:, b] + r[:, a] * ui[:, b] - 2 * r[:, a] * r[:, b] * rui)
                   + YG12 * (uj[:, a] * r[:, b] + r[:, a] * uj[:, b] - 2 * r[:, a] * r[:, b] * ruj)
                   + YH11 * (r[:, a] * ewi[:, b] + ewi[:, a] * r[:, b])
                   + YH12 * (r[:, a] * ewj[:, b] + ewj[:, a] * r[:, b]))
    out = np.zeros((N, 5))
    scatter_add(out, i, S)
    return -out.ravel()


def rse(pos, shear_rate, L, xy, rows, tdist, tvals, ori=None, b2mask=None, B2=0.0):
    """R_SE : E (Lubrication_RSE_kernel, Lubrication.cu:953-1230), pairs with r^2 < 16."""
    N = len(pos)
    E = strain_tensor(shear_rate, N, ori, b2mask, B2)
    i, j, r, dist = _lub_pairs(pos, L, xy, rows, 16.0)
    c = res_interp(dist, 16, 6, tdist, tvals)
    XM11, XM12, YM11, YM12, ZM11, ZM12 = c.T
    Eri = np.einsum("pab,pb->pa", E[i], r)
    Erj = np.einsum("pab,pb->pa", E[j], r)
    rEri = np.einsum("pa,pa->p", r, Eri)
    rErj = np.einsum("pa,pa->p", r, Erj)
    S = np.zeros((len(i), 5))
    for k, (a, b) in enumerate(_SAB):
        dab = 1.0 if a == b else 0.0
        P = r[:, a] * r[:, b] - dab / 3.0
        S[:, k] = (1.5 * XM11 * P * rEri + 1.5 * XM12 * P * rErj
                   + 0.5 * YM11 * (2 * r[:, a] * Eri[:, b] + 2 * r[:, b] * Eri[:, a] - 4 * rEri * r[:, a] * r[:, b])
                   + 0.5 * YM12 * (2 * r[:, a] * Erj[:, b] + 2 * r[:, b] * Erj[:, a] - 4 * rErj * r[:, a] * r[:, b])
                   + 0.5 * ZM11 * (2 * E[i][:, a, b] + (dab + r[:, a] * r[:, b]) * rEri
                                   - 2 * r[:, a] * Eri[:, b] - 2 * r[:, b] * Eri[:, a])
                   + 0.5 * ZM12 * (2 * E[j][:, a, b] + (dab + r[:, a] * r[:, b]) * rErj
                                   - 2 * r[:, a] * Erj[:, b] - 2 * r[:, b] * Erj[:, a]))
    out = np.zeros((N, 5))
    scatter_add(out, i, S)
    return out.ravel()


# ------------------------------------------------------------ saddle system
class Problem:
    """Everything the oracle needs about one configuration."""

    def __init__(self, pos, L, xy=0.0, xi=0.5, error=1e-3, max_strain=0.5, table=None, rlub=4.0, rp=2.1,
                 pi_typo=True, rows=None):
        self.pos = xyz(pos)
        self.N = len(self.pos)
        self.L = tuple(float(v) for v in L)
        self.xy = float(xy)
        self.xi = xi
        self.gp = grid_params(xi, error, max_strain, self.L)
        if table is None:
            raise ValueError("an Ewald table (reference golden or harness) is required")
        self.table, self.self_x, self.self_y, self.ewald_cut, self.ewald_n = table
        self.rows = rows if rows is not None else neighbor_list(self.pos, self.L, self.xy, self.ewald_cut + 0.4)
        self.tdist, self.tvals = resistance_table()
        self.rlub, self.rp = rlub, rp
        self.pi_typo = pi_typo

    def mobility(self, genF, parts=3):
        return mobility(self.pos, genF, self.L, self.xy, self.gp, self.xi, self.rows, self.table, self.self_x,
                        self.self_y, self.ewald_cut, self.ewald_n, parts, self.pi_typo)

    def rfu(self, U6):
        return rfu(self.pos, U6, self.L, self.xy, self.rows, self.tdist, self.tvals, self.rlub)

    def saddle_multiply(self, x):
        """Saddle_Multiply (Saddle.cu:80-151)."""
        N = self.N
        b = np.zeros(17 * N)
        b[: 11 * N] = self.mobility(x[: 11 * N])
        b[: 6 * N] += x[11 * N:]
        b[11 * N:] = x[: 6 * N] - self.rfu(x[11 * N:])
        return b

    def dense_saddle(self):
        N = self.N
        A = np.zeros((17 * N, 17 * N))
        for k in range(17 * N):
            e = np.zeros(17 * N)
            e[k] = 1.0
            A[:, k] = self.saddle_multiply(e)
        return A

    def solve(self, rhs, tol=1e-12):
        """Converged saddle solution: dense LU for small N, else FP64 GMRES with the
        block preconditioner of Saddle.cu:171-264 built on the exact (R_FU^pruned + D)^-1
        (sparse LU), iterated until the true residual is below tol."""
        if self.N <= 150:
            return np.linalg.solve(self.dense_saddle(), rhs)
        import scipy.sparse.linalg as sla
        N = self.N
        n = 17 * N
        lu = sla.splu(pruned_rfu_sparse(self.pos, self.L, self.xy, self.tdist, self.tvals, rows=self.rows,
                                        rp=self.rp).tocsc())

        def pc(b):
            y = lu.solve(b[: 6 * N] - b[11 * N:])
            x = b.copy()
            x[: 6 * N] = b[: 6 * N] - y
            x[11 * N:] = y
            return x

        A = sla.LinearOperator((n, n), matvec=self.saddle_multiply, dtype=np.float64)
        M = sla.LinearOperator((n, n), matvec=pc, dtype=np.float64)
        x = np.zeros(n)
        bn = np.linalg.norm(rhs)
        for _ in range(5):
            r = rhs - self.saddle_multiply(x)
            if np.linalg.norm(r) <= tol * bn:
                break
            dx, info = sla.gmres(A, r, M=M, rtol=tol * bn / max(np.linalg.norm(r), 1e-300), restart=200,
                                 maxiter=10)
            x = x + dx
        assert np.linalg.norm(rhs - self.saddle_multiply(x)) <= 10 * tol * bn
        return x

    def velocity(self, shear_rate, ndsr=0.1, k_n=1e4, kappa=20.0, beta=0.0, epsq=1e-5, tol=1e-10):
        """Integrator_ComputeVelocity (Integrator.cu:744-938) at kT = 0 without active
        terms: right-hand side from the interparticle force (Helper_Stokes.cu:65-172),
        the imposed strain (Helper_Integrator.cu:114-158) and R_FE:E
        (Lubrication.cu:350-608); the saddle solution; then U (6N) and the stresslet
        S = S^ff - R_SU U + R_SE:E (Integrator.cu:881-932, 5N).  Returns U, S, F."""
        N = self.N
        F = pair_force(self.pos, self.L, self.xy, self.rows, ndsr=ndsr, k_n=k_n, kappa=kappa, beta=beta, epsq=epsq)
        rhs = strain_rhs(shear_rate, N)
        rhs[11 * N:] -= F
        rhs[11 * N:] += rfe(self.pos, shear_rate, self.L, self.xy, self.rows, self.tdist, self.tvals, rlub=self.rlub)
        x = self.solve(rhs, tol)
        U = x[11 * N:]
        S = x[6 * N:11 * N] + rsu(self.pos, U, self.L, self.xy, self.rows, self.tdist, self.tvals, rlub=self.rlub) \
            + rse(self.pos, shear_rate, self.L, self.xy, self.rows, self.tdist, self.tvals)
        return U, S, F


def rcm(rows):
    """Reverse Cuthill-McKee as genrcm (rcm.cpp:1009): pseudo-peripheral root,
    breadth-first with new neighbours (all but the first) by increasing degree,
    reversed per component.  rows: adjacency per node (self loops allowed).  perm[new] = old."""
    n = len(rows)
    mask = np.ones(n, bool)
    perm = []

    def levels(root):
        order = [root]
        mask[root] = False
        starts = [0]
        lb = 0
        while True:
            le = len(order)
            for v in order[lb:le]:
                for u in rows[v]:
                    if mask[u]:
                        mask[u] = False
                        order.append(int(u))
            if len(order) == le:
                break
            starts.append(le)
            lb = le
        for v in order:
            mask[v] = True
        return order, starts

    for s in range(n):
        if not mask[s]:
            continue
        root = s
        order, starts = levels(root)
        nl, cs = len(starts), len(order)
        if nl > 1 and nl != cs:
            while True:
                ls = starts[-1]
                mindeg = cs
                root = order[ls]
                for v in order[ls:]:
                    d = int(sum(mask[u] for u in rows[v]))
                    if d < mindeg:
                        root, mindeg = v, d
                o2, s2 = levels(root)
                if len(s2) <= nl:
                    break
                nl = len(s2)
                order, starts = o2, s2
                if cs <= nl:
                    break
        order, _ = levels(root)
        deg = {v: int(sum(mask[u] for u in rows[v])) for v in order}
        comp = [root]
        mask[root] = False
        head = 0
        while head < len(comp):
            v = comp[head]
            head += 1
            new = []
            for u in rows[v]:
                if mask[u]:
                    mask[u] = False
                    new.append(int(u))
            # Stable insertion by degree over all but the first new neighbour:
            # the reference's loop (rcm.cpp, `while ( fnbr < l )`) never moves
            # the first one.
            new = new[:1] + sorted(new[1:], key=lambda x: deg[x])
            comp.extend(new)
        perm.extend(comp[::-1])
    return np.array(perm, np.int64)


def pruned_rfu_dense(pos, L, xy, rows, tdist, tvals, rp=2.1, relaxer=1.0):
    """Pruned R_FU plus relaxer * {1,1,1,4/3,4/3,4/3} on the diagonal, dense 6N x 6N
    (Precondition_RFU_kernel, Precondition.cu:530-836; AddIdentity,
    Helper_Precondition.cu:535-580).  Also returns the particle graph rows."""
    pos = xyz(pos)
    N = len(pos)
    prow = []
    for i in range(N):
        d = min_image(pos[i] - pos[np.asarray(rows[i], np.int64)], L, xy)
        keep = np.einsum("ij,ij->i", d, d) < rp * rp
        prow.append(np.sort(np.concatenate([[i], np.asarray(rows[i], np.int64)[keep]])))
    A = np.zeros((6 * N, 6 * N))
    for i in range(N):
        for j in prow[i]:
            if j == i:
                continue
            R = min_image32((pos[j] - pos[i]).astype(F32)[None], L, xy)[0]
            dist = np.sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2])
            R = R.astype(np.float64)
            c = res_interp(np.array([dist]), 0, 10, tdist, tvals, mode="precond")[0]
            XA11, XA12, YA11, YA12, YB11, YB12, XC11, XC12, YC11, YC12 = c
            r = R / dist
            rr = np.outer(r, r)
            Im = np.eye(3) - rr
            eps = np.array([[0, r[2], -r[1]], [-r[2], 0, r[0]], [r[1], -r[0], 0]])
            bi, bj = 6 * i, 6 * j
            A[bi:bi + 3, bj:bj + 3] = XA12 * rr + YA12 * Im
            A[bi:bi + 3, bj + 3:bj + 6] = YB12 * eps
            A[bi + 3:bi + 6, bj:bj + 3] = YB12 * eps
            A[bi + 3:bi + 6, bj + 3:bj + 6] = XC12 * rr + YC12 * Im
            A[bi:bi + 3, bi:bi + 3] += XA11 * rr + YA11 * Im
            A[bi:bi + 3, bi + 3:bi + 6] += -YB11 * eps
            A[bi + 3:bi + 6, bi:bi + 3] += YB11 * eps
            A[bi + 3:bi + 6, bi + 3:bi + 6] += XC11 * rr + YC11 * Im
    d = np.tile([1.0, 1.0, 1.0, float(F32(1.33333333)), float(F32(1.33333333)), float(F32(1.33333333))], N)
    A[np.arange(6 * N), np.arange(6 * N)] += relaxer * d
    return A, prow


def pruned_pairs(pos, L, xy, rows=None, rp=2.1):
    """Directed pairs (i, j), i != j, of the pruned graph: float64 minimum-image
    distance below rp (Precondition_GetPrunedNneigh_kernel, Precondition.cu:443).
    Candidates come from `rows`, or from a periodic k-d tree for untilted boxes."""
    x = xyz(pos)
    if rows is None:
        from scipy.spatial import cKDTree
        if xy != 0.0:
            raise ValueError("k-d tree candidates need an untilted box; pass rows")
        Lb = np.asarray(L, np.float64)
        pr = cKDTree(np.mod(x + Lb / 2, Lb), boxsize=Lb).query_pairs(rp + 1e-3, output_type="ndarray")
        i = np.concatenate([pr[:, 0], pr[:, 1]]).astype(np.int64)
        j = np.concatenate([pr[:, 1], pr[:, 0]]).astype(np.int64)
    else:
        i, j = pair_arrays(rows)
    d = min_image(x[i] - x[j], L, xy)
    keep = np.einsum("ij,ij->i", d, d) < rp * rp
    i, j = i[keep], j[keep]
    o = np.lexsort((j, i))
    return i[o], j[o]


def pruned_rfu_sparse(pos, L, xy, tdist, tvals, rows=None, rp=2.1, relaxer=1.0):
    """pruned_rfu_dense as a SciPy CSR matrix, vectorised for large N."""
    import scipy.sparse as sp
    x = xyz(pos)
    N = len(x)
    i, j = pruned_pairs(pos, L, xy, rows, rp)
    R = min_image32((x[j] - x[i]).astype(F32), L, xy)
    dist = np.sqrt(R[:, 0] * R[:, 0] + R[:, 1] * R[:, 1] + R[:, 2] * R[:, 2])
    R = R.astype(np.float64)
    c = res_interp(dist, 0, 10, tdist, tvals, mode="precond")
    XA11, XA12, YA11, YA12, YB11, YB12, XC11, XC12, YC11, YC12 = c.T
    r = R / dist.astype(np.float64)[:, None]
    rr = r[:, :, None] * r[:, None, :]
    Im = np.eye(3)[None] - rr
    eps = np.zeros((len(r), 3, 3))
    eps[:, 0, 1], eps[:, 0, 2] = r[:, 2], -r[:, 1]
    eps[:, 1, 0], eps[:, 1, 2] = -r[:, 2], r[:, 0]
    eps[:, 2, 0], eps[:, 2, 1] = r[:, 1], -r[:, 0]
    w = lambda a: a[:, None, None]
    off = np.zeros((len(r), 6, 6))
    off[:, :3, :3] = w(XA12) * rr + w(YA12) * Im
    off[:, :3, 3:] = w(YB12) * eps
    off[:, 3:, :3] = w(YB12) * eps
    off[:, 3:, 3:] = w(XC12) * rr + w(YC12) * Im
    slf = np.zeros((len(r), 6, 6))
    slf[:, :3, :3] = w(XA11) * rr + w(YA11) * Im
    slf[:, :3, 3:] = -w(YB11) * eps
    slf[:, 3:, :3] = w(YB11) * eps
    slf[:, 3:, 3:] = w(XC11) * rr + w(YC11) * Im
    diag = np.zeros((N, 6, 6))
    scatter_add(diag, i, slf)
    d = np.array([1.0, 1.0, 1.0] + [float(F32(1.33333333))] * 3)
    diag[:, np.arange(6), np.arange(6)] += relaxer * d
    bi = np.concatenate([i, np.arange(N)])
    bj = np.concatenate([j, np.arange(N)])
    vals = np.concatenate([off, diag])
    rows_ = (6 * bi[:, None, None] + np.arange(6)[None, :, None]) * np.ones((1, 1, 6), np.int64)
    cols_ = (6 * bj[:, None, None] + np.arange(6)[None, None, :]) * np.ones((1, 6, 1), np.int64)
    return sp.csr_matrix((vals.ravel(), (rows_.ravel(), cols_.ravel())), shape=(6 * N, 6 * N))


def spai_sets(A_bsr, N, cap=32):
    """Two-hop sets as the CUDA path builds them: the particle, its pruned
    neighbours in index order, then new members of their lists in order,
    truncated at cap."""
    sets = []
    rows = [A_bsr.indices[A_bsr.indptr[k]:A_bsr.indptr[k + 1]] for k in range(N)]
    for c in range(N):
        S = [c] + [int(k) for k in rows[c] if k != c][: cap - 1]
        for k in S[1:len(S)]:
            for q in rows[k]:
                q = int(q)
                if q not in S and len(S) < cap:
                    S.append(q)
        sets.append(S)
    return sets


def spai2(A, N, cap=32):
    """Right sparse approximate inverse on the two-hop sets: column c of G is
    X_c with (A^2)[S_c, S_c] X_c = A[S_c, c] (FP64 normal equations), block
    (s, c) kept where c is in the set of s (as the CUDA path stores it in row
    s).  Returns a SciPy CSR matrix."""
    import scipy.sparse as sp
    Ab = sp.bsr_matrix(A, blocksize=(6, 6))
    Ab.sort_indices()
    sets = spai_sets(Ab, N, cap)
    member = [set(S) for S in sets]
    Ac = A.tocsc()
    rows, cols, vals = [], [], []
    r, q = np.meshgrid(np.arange(6), np.arange(6), indexing="ij")
    for c, S in enumerate(sets):
        idx = np.concatenate([np.arange(6 * s, 6 * s + 6) for s in S])
        As = Ac[:, idx].toarray()
        X = np.linalg.solve(As.T @ As, As[6 * c:6 * c + 6].T)
        for a, s in enumerate(S):
            if c not in member[s]:
                continue
            rows.append((6 * s + r).ravel())
            cols.append((6 * c + q).ravel())
            vals.append(X[6 * a:6 * a + 6].ravel())
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=A.shape)


def spai2_columns(A, N, cols, cap=32):
    """The blocks of spai2 in the given block columns only: {(s, c): 6x6}
    for c in cols and every s whose set holds c (same rule as spai2)."""
    import scipy.sparse as sp
    Ab = sp.bsr_matrix(A, blocksize=(6, 6))
    Ab.sort_indices()
    sets = spai_sets(Ab, N, cap)
    Ac = A.tocsc()
    out = {}
    for c in cols:
        S = sets[c]
        idx = np.concatenate([np.arange(6 * s, 6 * s + 6) for s in S])
        As = Ac[:, idx].toarray()
        X = np.linalg.solve(As.T @ As, As[6 * c:6 * c + 6].T)
        for a, s in enumerate(S):
            if c in sets[s]:
                out[(s, c)] = X[6 * a:6 * a + 6]
    return out


def ichol0_dense(A, pattern):
    """Scalar IC(0) restricted to `pattern` (boolean), FP64.  Returns L or None on a non-positive pivot."""
    n = len(A)
    L = np.where(pattern, A, 0.0).copy()
    L = np.tril(L)
    for k in range(n):
        if not L[k, k] > 0:
            return None
        L[k, k] = np.sqrt(L[k, k])
        col = np.nonzero(pattern[k + 1:, k])[0] + k + 1
        L[col, k] /= L[k, k]
        for j in col:
            rows_ = col[col >= j]
            rows_ = rows_[pattern[rows_, j]]  # zero fill: update only entries of the pattern
            L[rows_, j] -= L[rows_, k] * L[j, k]
    return L


def saddle_precond(b, G, N):
    """Saddle_Preconditioner (Saddle.cu:171-264) with G ~ (R_FU^pruned + relaxer D)^-1."""
    b = np.asarray(b, np.float64)
    y = G @ (b[: 6 * N] - b[11 * N:])
    x = b.copy()
    x[: 6 * N] = b[: 6 * N] - y
    x[11 * N:] = y
    return x


# ------------------------------------------------------------ forces, motion
def pair_force(pos, L, xy, rows, ndsr=0.1, k_n=1e4, kappa=20.0, beta=0.0, epsq=1e-5, T_ext=0.0):
    """Repulsion + van der Waals + collision force and z torque (Stokes_SetForce_manually_kernel,
    Helper_Stokes.cu:65-172)."""
    p32 = np.asarray(pos, F32)[:, :3]
    N = len(p32)
    i, j = pair_arrays(rows)
    # single-precision separation and distance, as the kernel: near contact the
    # collision term k_n |gap| resolves the gap only to float32
    R32 = min_image32(p32[j] - p32[i], L, xy)
    d2 = R32[:, 0] * R32[:, 0] + R32[:, 1] * R32[:, 1] + R32[:, 2] * R32[:, 2]
    R = R32.astype(np.float64)
    d32 = np.sqrt(d2)
    dist = d32.astype(np.float64)
    # contact radius and gap in single precision as the kernel (2 + sqrt(epsq),
    # dist - rcol): at k_n = 1e4 the rounding of rcol is visible in the force
    rcol32 = F32(2.0) + F32(np.sqrt(F32(epsq)))
    F0 = 1.0 / ndsr
    H = F0 * beta
    gap = (d32 - rcol32).astype(np.float64)
    mag = np.zeros_like(dist)
    m1 = (gap >= 0) & (dist <= 2.0 + 10.0 / kappa)
    mag[m1] = H / (12.0 * (gap[m1] ** 2 + epsq)) - F0 * np.exp(-kappa * gap[m1])
    m2 = gap < 0
    mag[m2] = H / (12.0 * epsq) - F0 - k_n * np.abs(gap[m2])
    out = np.zeros((N, 6))
    scatter_add(out[:, :3], i, mag[:, None] * R / dist[:, None])
    out[:, 5] = T_ext
    return out.ravel()


def strain_rhs(shear_rate, N, ori=None, b2mask=None, B2=0.0):
    """Imposed strain minus the active strain in the stresslet rows of the
    right-hand side (Integrator_AddStrainRate_kernel, Helper_Integrator.cu:114-158)."""
    b = np.zeros(17 * N)
    e = b[6 * N: 11 * N].reshape(N, 5)
    e[:, 1] += shear_rate
    if B2 != 0.0 and ori is not None:
        p = np.asarray(ori, np.float64)
        m = np.ones(N) if b2mask is None else np.asarray(b2mask, np.float64)
        b2 = -0.6 * B2 * m
        e[:, 0] -= b2 * (p[:, 0] ** 2 - p[:, 2] ** 2)
        e[:, 1] -= b2 * 2 * p[:, 0] * p[:, 1]
        e[:, 2] -= b2 * 2 * p[:, 0] * p[:, 2]
        e[:, 3] -= b2 * 2 * p[:, 1] * p[:, 2]
        e[:, 4] -= b2 * (p[:, 1] ** 2 - p[:, 2] ** 2)
    return b


def wrap(p, img, L, xy):
    """HOOMD BoxDim::wrap with an xy tilt: one image shift per axis, x then y then z."""
    p = p.copy()
    img = img.copy()
    Lx, Ly, Lz = L
    tilt = xy * p[:, 1]
    hi = p[:, 0] >= Lx / 2 + tilt
    lo = p[:, 0] < -Lx / 2 + tilt
    p[hi, 0] -= Lx
    img[hi, 0] += 1
    p[lo & ~hi, 0] += Lx
    img[lo & ~hi, 0] -= 1
    hi = p[:, 1] >= Ly / 2
    lo = (p[:, 1] < -Ly / 2) & ~hi
    p[hi, 1] -= Ly
    p[hi, 0] -= Ly * xy
    img[hi, 1] += 1
    p[lo, 1] += Ly
    p[lo, 0] += Ly * xy
    img[lo, 1] -= 1
    hi = p[:, 2] >= Lz / 2
    lo = (p[:, 2] < -Lz / 2) & ~hi
    p[hi, 2] -= Lz
    img[hi, 2] += 1
    p[lo, 2] += Lz
    img[lo, 2] -= 1
    return p, img


def euler_shear(pos, ori, pos_gb, vel, image, L, xy, dt, shear_rate, B1=0.0, b1mask=None, noise=None):
    """Explicit Euler with simple shear and director rotation
    (Integrator_ExplicitEuler_Shear_kernel, Integrator.cu:126-228)."""
    pos = xyz(pos)
    N = len(pos)
    V = np.asarray(vel, np.float64)[: 6 * N].reshape(N, 6)
    p = pos[:, :3].copy()
    v = V[:, :3].copy()
    w = V[:, 3:].copy()
    v[:, 0] += shear_rate * p[:, 1]
    w[:, 2] -= shear_rate / 2.0
    if noise is not None:
        w += np.asarray(noise, np.float64)
    aw = np.linalg.norm(w, axis=1)
    rot = aw > 1e-6
    q0 = np.ones(N)
    qv = np.zeros((N, 3))
    ang = aw * dt
    q0[rot] = np.cos(ang[rot] / 2)
    qv[rot] = w[rot] / aw[rot, None] * np.sin(ang[rot] / 2)[:, None]
    pv = np.asarray(ori, np.float64)
    m = np.ones(N) if b1mask is None else np.asarray(b1mask, np.float64)
    v -= (-2.0 / 3.0 * B1 * m)[:, None] * pv
    gb = np.asarray(pos_gb, np.float64).copy()
    gb[:, 0] += (v[:, 0] - shear_rate * p[:, 1] + shear_rate * gb[:, 1]) * dt
    gb[:, 1] += v[:, 1] * dt
    gb[:, 2] += v[:, 2] * dt
    p, img = wrap(p + v * dt, np.asarray(image, np.int64), L, xy)
    qq = np.einsum("ij,ij->i", qv, qv)
    qp = np.einsum("ij,ij->i", qv, pv)
    pn = (q0 * q0 - qq)[:, None] * pv + 2 * qp[:, None] * qv + 2 * q0[:, None] * np.cross(qv, pv)
    pn /= np.linalg.norm(pn, axis=1, keepdims=True)
    return p, pn, gb, img


# --------------------------------------------------- friction, Runge-Kutta
def friction_table(tdist, tvals, h0, alpha):
    """Stokes::setFriction TYPE1 (Stokes.cc:1132-1191): for gaps h = r - 2 <= h0
    add alpha_k (2 h^2/h0^3 - 3 h/h0^2 + 1/h) in magnitude to YA11, YA12, YB11,
    YB12, YC11, YC12 (entries 3, 4, 5, 6, 9, 10).  Single-precision h and
    powers of h0, the bracket in double, the sum rounded to single precision,
    as the reference's mix of float variables and double literals."""
    vals = np.array(tvals, np.float32, copy=True).reshape(-1, 22)
    h0 = F32(h0)
    h02 = F32(h0 * h0)
    h03 = F32(h0 * h02)
    slots = (3, 4, 5, 6, 9, 10)
    signs = (1, -1, -1, 1, 1, 1)
    for i, d in enumerate(np.asarray(tdist, np.float32)):
        h = F32(float(d) - 2.0)
        if not h <= h0:
            continue
        h2 = F32(h * h)
        bracket = 2.0 / float(h03) * float(h2) - 3.0 / float(h02) * float(h) + 1.0 / float(h)
        for a, slot, sg in zip(alpha, slots, signs):
            add = F32(float(F32(a)) * bracket)
            vals[i, slot] = F32(vals[i, slot] + add) if sg > 0 else F32(vals[i, slot] - add)
    return vals


def _rotate(pv, w, t):
    aw = np.linalg.norm(w, axis=1)
    rot = aw > 1e-6
    q0 = np.ones(len(pv))
    qv = np.zeros_like(pv)
    q0[rot] = np.cos(aw[rot] * t / 2)
    qv[rot] = w[rot] / aw[rot, None] * np.sin(aw[rot] * t / 2)[:, None]
    qq = np.einsum("ij,ij->i", qv, qv)
    qp = np.einsum("ij,ij->i", qv, pv)
    pn = (q0 * q0 - qq)[:, None] * pv + 2 * qp[:, None] * qv + 2 * q0[:, None] * np.cross(qv, pv)
    return pn / np.linalg.norm(pn, axis=1, keepdims=True)


def rk_stage1(pos, ori, pos_gb, vel, dt, shear_rate, B1=0.0, b1mask=None, noise=None):
    """Integrator_ExplicitEuler1_Shear_kernel (Integrator.cu:232-330): the
    unwrapped predictor, the director rotated by dt, half a step of pos_gb."""
    p = xyz(pos).copy()
    N = len(p)
    V = np.asarray(vel, np.float64)[: 6 * N].reshape(N, 6)
    v, w = V[:, :3].copy(), V[:, 3:].copy()
    v[:, 0] += shear_rate * p[:, 1]
    w[:, 2] -= shear_rate / 2.0
    if noise is not None:
        w += np.asarray(noise, np.float64)
    pv = np.asarray(ori, np.float64)
    m = np.ones(N) if b1mask is None else np.asarray(b1mask, np.float64)
    v -= (-2.0 / 3.0 * B1 * m)[:, None] * pv
    gb = np.asarray(pos_gb, np.float64).copy()
    gb[:, 0] += (v[:, 0] - shear_rate * p[:, 1] + shear_rate * gb[:, 1]) * 0.5 * dt
    gb[:, 1] += v[:, 1] * 0.5 * dt
    gb[:, 2] += v[:, 2] * 0.5 * dt
    return p + v * dt, _rotate(pv, w, dt), gb


def rk_stage2(pos, ori, pos_star, ori_star, pos_gb, vel, image, L, xy, dt, shear_rate, B1=0.0, b1mask=None,
              noise=None, c1=0.5, c2=0.5, c3=0.5):
    """Integrator_RK_Shear_kernel (Integrator.cu:333-438)."""
    p = c1 * xyz(pos) + c2 * xyz(pos_star)
    N = len(p)
    V = np.asarray(vel, np.float64)[: 6 * N].reshape(N, 6)
    v, w = V[:, :3].copy(), V[:, 3:].copy()
    v[:, 0] += shear_rate * p[:, 1]
    w[:, 2] -= shear_rate / 2.0
    if noise is not None:
        w += np.asarray(noise, np.float64)
    pv = c1 * np.asarray(ori, np.float64) + c2 * np.asarray(ori_star, np.float64)
    pv /= np.linalg.norm(pv, axis=1, keepdims=True)
    m = np.ones(N) if b1mask is None else np.asarray(b1mask, np.float64)
    v -= (-2.0 / 3.0 * B1 * m)[:, None] * pv
    gb = np.asarray(pos_gb, np.float64).copy()
    gb[:, 0] += (v[:, 0] - shear_rate * p[:, 1] + shear_rate * gb[:, 1]) * 0.5 * dt
    gb[:, 1] += v[:, 1] * 0.5 * dt
    gb[:, 2] += v[:, 2] * 0.5 * dt
    pn, img = wrap(p + v * dt * c3, np.asarray(image, np.int64), L, xy)
    return pn, _rotate(pv, w, dt * c3), gb, img
