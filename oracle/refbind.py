"""ctypes binding of oracle/_ref/libfsdref.so (reference pieces built for the host).

Test infrastructure only.  ``available()`` is False when the library has not
been built (for example on machines without the reference checkout); callers
then use the committed golden fixtures instead.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libfsdref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(LIB))
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


F = C.c_float


def setparams(xi, error, max_strain, L):
    oi = np.zeros(4, np.int32)
    of = np.zeros(6, np.float32)
    lib().ref_setparams(F(xi), F(error), F(max_strain), F(L[0]), F(L[1]), F(L[2]), _p(oi), _p(of))
    return dict(Nx=int(oi[0]), Ny=int(oi[1]), Nz=int(oi[2]), P=int(oi[3]), ewald_cut=float(of[0]),
                gauss_m=float(of[1]), eta=float(of[2]), hx=float(of[3]), hy=float(of[4]), hz=float(of[5]))


def ewald_table(xi, error):
    self2 = np.zeros(2, np.float32)
    cut = C.c_float()
    n = C.c_int()
    nR = lib().ref_ewald_table(F(xi), F(error), None, _p(self2), C.byref(cut), C.byref(n))
    tab = np.zeros((2 * nR, 4), np.float32)
    lib().ref_ewald_table(F(xi), F(error), _p(tab), _p(self2), C.byref(cut), C.byref(n))
    return tab, float(self2[0]), float(self2[1]), float(cut.value), int(n.value)


def gridk(N3, L, xy, xi, eta):
    Nx, Ny, Nz = N3
    out = np.zeros((Nx * Ny * Nz, 4), np.float32)
    lib().ref_gridk(_p(out), Nx, Ny, Nz, F(L[0]), F(L[1]), F(L[2]), F(xy), F(xi), F(eta))
    return out


def green(grids11: np.ndarray, gk: np.ndarray):
    """grids11: complex64 (11, G) in order X Y Z XX XY XZ YX YY YZ ZX ZY; modified copy returned."""
    g = np.ascontiguousarray(grids11.astype(np.complex64))
    lib().ref_green(_p(g), _p(np.ascontiguousarray(gk, np.float32)), g.shape[1])
    return g


def _nl(nlist_rows):
    nn = np.array([len(r) for r in nlist_rows], np.uint32)
    head = np.zeros(len(nlist_rows), np.uint32)
    head[1:] = np.cumsum(nn)[:-1]
    flat = np.concatenate([np.asarray(r, np.uint32) for r in nlist_rows]) if nn.sum() else np.zeros(1, np.uint32)
    return nn, np.ascontiguousarray(flat, np.uint32), head


def realspace(pos4, force4, couplet8, nlist_rows, L, xy, xi, table, self_x, self_y, ewald_cut, ewald_n, ewald_dr=1e-3):
    N = len(pos4)
    nn, flat, head = _nl(nlist_rows)
    vel = np.zeros((N, 4), np.float32)
    delu = np.zeros((2 * N, 4), np.float32)
    c4 = np.ascontiguousarray(couplet8.reshape(2 * N, 4), np.float32)
    lib().ref_realspace(_p(np.ascontiguousarray(pos4, np.float32)), _p(vel), _p(delu),
                        _p(np.ascontiguousarray(force4, np.float32)), _p(c4), N, F(xi),
                        _p(np.ascontiguousarray(table, np.float32)), F(self_x), F(self_y), F(ewald_cut), ewald_n,
                        F(ewald_dr), F(L[0]), F(L[1]), F(L[2]), F(xy), _p(nn), _p(flat), _p(head))
    return vel, delu.reshape(N, 8)


def ts2c(ts8):
    N = len(ts8)
    c = np.zeros((2 * N, 4), np.float32)
    lib().ref_ts2c(_p(c), _p(np.ascontiguousarray(ts8.reshape(2 * N, 4), np.float32)), N)
    return c.reshape(N, 8)


def d2we(delu8):
    N = len(delu8)
    o = np.zeros((2 * N, 4), np.float32)
    lib().ref_d2we(_p(np.ascontiguousarray(delu8.reshape(2 * N, 4), np.float32)), _p(o), N)
    return o.reshape(N, 8)


def _table_like_reference(tdist, tvals):
    """The reference's table buffers: values in a 32000-float array zero past
    entry 22000 (Stokes_ResistanceTable.cc:46-47, HOOMD zero-fills GPUArrays)
    and distances in an allocation padded to 256 bytes.  Pairs with
    3.9978 <= r < 4 index one row past the table (Lubrication.cu:193-200) and
    read those zeros."""
    d = np.zeros(1024, np.float32)
    d[:1000] = np.asarray(tdist, np.float32).ravel()
    v = np.zeros(32000, np.float32)
    v[:22000] = np.asarray(tvals, np.float32).ravel()
    return d, v


def _lub_common(pos4, nlist_rows, L, xy):
    nn, flat, head = _nl(nlist_rows)
    return np.ascontiguousarray(pos4, np.float32), nn, flat, head


def rfu(pos4, U6, nlist_rows, L, xy, tdist, tvals, rlub=4.0, tmin=1e-4, tdr=0.004305):
    tdist, tvals = _table_like_reference(tdist, tvals)
    N = len(pos4)
    pos, nn, flat, head = _lub_common(pos4, nlist_rows, L, xy)
    F6 = np.zeros(6 * N, np.float32)
    lib().ref_rfu(_p(F6), _p(np.ascontiguousarray(U6, np.float32)), _p(pos), N, F(L[0]), F(L[1]), F(L[2]), F(xy),
                  _p(nn), _p(flat), _p(head), _p(tdist), _p(tvals), F(tmin), F(tdr), F(rlub))
    return F6


def rfe(pos4, shear_rate, nlist_rows, L, xy, tdist, tvals, ori=None, b2mask=None, B2=0.0, rlub=4.0, tmin=1e-4,
        tdr=0.004305):
    tdist, tvals = _table_like_reference(tdist, tvals)
    N = len(pos4)
    pos, nn, flat, head = _lub_common(pos4, nlist_rows, L, xy)
    ori = np.zeros((N, 3), np.float32) if ori is None else np.ascontiguousarray(ori, np.float32)
    b2mask = np.ones(N, np.float32) if b2mask is None else np.ascontiguousarray(b2mask, np.float32)
    F6 = np.zeros(6 * N, np.float32)
    lib().ref_rfe(_p(F6), F(shear_rate), _p(pos), F(B2), _p(b2mask), _p(ori), N, F(L[0]), F(L[1]), F(L[2]), F(xy),
                  _p(nn), _p(flat), _p(head), _p(tdist), _p(tvals), F(tmin), F(tdr), F(rlub))
    return F6


def rsu(pos4, U6, nlist_rows, L, xy, tdist, tvals, rlub=4.0, tmin=1e-4, tdr=0.004305):
    tdist, tvals = _table_like_reference(tdist, tvals)
    N = len(pos4)
    pos, nn, flat, head = _lub_common(pos4, nlist_rows, L, xy)
    S = np.zeros(5 * N, np.float32)
    lib().ref_rsu(_p(S), _p(np.ascontiguousarray(U6, np.float32)), _p(pos), N, F(L[0]), F(L[1]), F(L[2]), F(xy),
                  _p(nn), _p(flat), _p(head), _p(tdist), _p(tvals), F(tmin), F(tdr), F(rlub))
    return S


def rse(pos4, shear_rate, nlist_rows, L, xy, tdist, tvals, ori=None, b2mask=None, B2=0.0, tmin=1e-4, tdr=0.004305):
    tdist, tvals = _table_like_reference(tdist, tvals)
    N = len(pos4)
    pos, nn, flat, head = _lub_common(pos4, nlist_rows, L, xy)
    ori = np.zeros((N, 3), np.float32) if ori is None else np.ascontiguousarray(ori, np.float32)
    b2mask = np.ones(N, np.float32) if b2mask is None else np.ascontiguousarray(b2mask, np.float32)
    S = np.zeros(5 * N, np.float32)
    lib().ref_rse(_p(S), F(shear_rate), F(B2), _p(b2mask), _p(ori), N, _p(nn), _p(flat), _p(head), _p(pos),
                  F(L[0]), F(L[1]), F(L[2]), F(xy), _p(tdist), _p(tvals), F(tmin), F(tdr))
    return S


def pruned_nlist(pos4, nlist_rows, L, xy, rp=2.1):
    N = len(pos4)
    pos, nn, flat, head = _lub_common(pos4, nlist_rows, L, xy)
    nn_p = np.zeros(N, np.uint32)
    head_p = np.zeros(N + 1, np.uint32)
    nl_p = np.zeros(int(nn.sum()) + N + 1, np.uint32)
    nless = np.zeros(N, np.uint32)
    lib().ref_pruned_nlist(_p(pos), N, F(L[0]), F(L[1]), F(L[2]), F(xy), _p(nn), _p(flat), _p(head), F(rp),
                           _p(nn_p), _p(nl_p), _p(head_p), _p(nless))
    return [nl_p[head_p[i]: head_p[i] + nn_p[i]].copy() for i in range(N)], nless


def precond_coo(pos4, nlist_rows, L, xy, tdist, tvals, rp=2.1, tmin=1e-4, tdr=0.004305):
    tdist, tvals = _table_like_reference(tdist, tvals)
    """Pruned R_FU in COO as the reference assembles it (before the identity shift)."""
    N = len(pos4)
    rows, nless = pruned_nlist(pos4, nlist_rows, L, xy, rp)
    nn_p = np.array([len(r) for r in rows], np.uint32)
    head_p = np.zeros(N + 1, np.uint32)
    head_p[1:] = np.cumsum(nn_p)
    flat = np.concatenate(rows).astype(np.uint32)
    cap = 36 * int(nn_p.sum()) + 16 * N
    r = np.zeros(cap, np.int32)
    c = np.zeros(cap, np.int32)
    v = np.zeros(cap, np.float32)
    nnz = lib().ref_precond_rfu_coo(_p(np.ascontiguousarray(pos4, np.float32)), N, F(L[0]), F(L[1]), F(L[2]), F(xy),
                                    _p(nn_p), _p(flat), _p(head_p), _p(nless), _p(tdist), _p(tvals), F(tmin), F(tdr),
                                    F(rp), _p(r), _p(c), _p(v), cap)
    assert nnz > 0
    return r[:nnz], c[:nnz], v[:nnz], rows


def genrcm(rows):
    """Reference genrcm on the graph given by per-node adjacency rows; returns a 0-based perm (perm[new] = old)."""
    n = len(rows)
    adj_row = np.zeros(n + 1, np.int32)
    adj_row[1:] = np.cumsum([len(r) for r in rows])
    adj = (np.concatenate(rows).astype(np.int32) + 1) if adj_row[-1] else np.zeros(1, np.int32)
    adj_row = adj_row + 1
    perm = np.zeros(n, np.int32)
    lib().ref_genrcm(n, int(adj_row[-1] - 1), _p(adj_row), _p(np.ascontiguousarray(adj)), _p(perm))
    return perm - 1


def setforce(pos4, ori, nlist_rows, L, xy, ndsr=0.1, k_n=1e4, kappa=20.0, beta=0.0, epsq=1e-5, T_ext=0.0):
    N = len(pos4)
    pos, nn, flat, head = _lub_common(pos4, nlist_rows, L, xy)
    F6 = np.zeros(6 * N, np.float32)
    lib().ref_setforce(_p(pos), _p(np.ascontiguousarray(ori, np.float32)), _p(F6), N, _p(nn), _p(flat), _p(head),
                       F(ndsr), F(k_n), F(kappa), F(beta), F(epsq), F(T_ext), F(L[0]), F(L[1]), F(L[2]), F(xy))
    return F6


def add_strain_rate(b17, shear_rate, N, ori=None, b2mask=None, B2=0.0):
    b = np.ascontiguousarray(b17, np.float32).copy()
    ori = np.zeros((N, 3), np.float32) if ori is None else np.ascontiguousarray(ori, np.float32)
    b2mask = np.ones(N, np.float32) if b2mask is None else np.ascontiguousarray(b2mask, np.float32)
    lib().ref_add_strain_rate(_p(b), F(shear_rate), F(B2), _p(b2mask), _p(ori), N)
    return b


def euler_shear(pos4, ori, pos_gb, vel, image, L, xy, dt, shear_rate, B1=0.0, b1mask=None, noise=None):
    N = len(pos4)
    pos = np.ascontiguousarray(pos4, np.float32).copy()
    o = np.ascontiguousarray(ori, np.float32).copy()
    gb = np.ascontiguousarray(pos_gb, np.float32).copy()
    img = np.ascontiguousarray(image, np.int32).copy()
    b1mask = np.ones(N, np.float32) if b1mask is None else np.ascontiguousarray(b1mask, np.float32)
    noise = np.zeros((N, 3), np.float32) if noise is None else np.ascontiguousarray(noise, np.float32)
    lib().ref_euler_shear(_p(pos), _p(o), _p(gb), _p(np.ascontiguousarray(vel, np.float32)), F(B1), _p(b1mask),
                          _p(noise), _p(img), N, F(L[0]), F(L[1]), F(L[2]), F(xy), F(dt), F(shear_rate))
    return pos, o, gb, img


def euler(pos4, vel, image, L, xy, dt):
    N = len(pos4)
    out = np.zeros_like(np.ascontiguousarray(pos4, np.float32))
    img = np.ascontiguousarray(image, np.int32).copy()
    lib().ref_euler(_p(np.ascontiguousarray(pos4, np.float32)), _p(out), _p(np.ascontiguousarray(vel, np.float32)),
                    _p(img), N, F(L[0]), F(L[1]), F(L[2]), F(xy), F(dt))
    return out
