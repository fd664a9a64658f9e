"""The oracle restatement against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the reference compiled for the host),
and, when oracle/_ref has been built here, against the live reference on fresh
random inputs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import ewald_golden, golden, rows_from
from oracle import fsd_oracle as O
from oracle import refbind as R


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_grid_params_match_reference():
    for case in golden("setparams.json"):
        got = O.grid_params(case["xi"], case["error"], case["max_strain"], case["L"])
        ref = case["ref"]
        for k in ("Nx", "Ny", "Nz", "P"):
            assert got[k] == ref[k], (case, k)
        for k in ("ewald_cut", "gauss_m", "eta", "hx", "hy", "hz"):
            assert np.float32(got[k]) == np.float32(ref[k]), (case, k, got[k], ref[k])


def test_resistance_table_known_values():
    d, v = O.resistance_table()
    # Stokes_ResistanceTable.cc:56-59, 1058-1059 (first rows) and the zero last row.
    assert d[0] == np.float32(2.000100) and d[1] == np.float32(2.000101) and d[-1] == np.float32(4.0)
    assert v[0, 0] == np.float32(2500.839791) and v[0, 1] == np.float32(-2500.837257)
    assert np.all(v[-1] == 0)
    assert d[232] == np.float32(2.000997)


def test_self_terms_known_answer():
    # Stokes.cc:367-371 at xi = 0.5, a = 1.
    tab, sx, sy, cut, n = ewald_golden()
    xi = 0.5
    from math import erfc, exp, pi, sqrt
    assert abs(sx - (1 + 4 * sqrt(pi) * xi * erfc(2 * xi) - exp(-4 * xi * xi)) / (4 * sqrt(pi) * xi)) < 1e-6
    assert n == int(np.float32(cut) / np.float32(0.001) - 1)


@pytest.mark.parametrize("case", ["pairs_dilute.npz", "pairs_dense_sheared.npz"])
def test_lubrication_oracle_matches_reference(case):
    g = golden(case)
    pos, L, xy = g["pos"], tuple(g["L"]), float(g["xy"])
    rows = rows_from(g["nn"], g["flat"])
    td, tv = O.resistance_table()
    kw = dict(ori=g["ori"], b2mask=g["b2mask"], B2=float(g["B2"]))
    assert rel(O.rfu(pos, g["U6"], L, xy, rows, td, tv), g["rfu"]) < 2e-6
    assert rel(O.rfe(pos, float(g["shear_rate"]), L, xy, rows, td, tv, **kw), g["rfe"]) < 2e-6
    assert rel(O.rsu(pos, g["U6"], L, xy, rows, td, tv), g["rsu"]) < 2e-6
    assert rel(O.rse(pos, float(g["shear_rate"]), L, xy, rows, td, tv, **kw), g["rse"]) < 2e-6


@pytest.mark.parametrize("case", ["pairs_dilute.npz", "pairs_dense_sheared.npz"])
def test_realspace_oracle_matches_reference(case):
    g = golden(case)
    pos, L, xy = g["pos"], tuple(g["L"]), float(g["xy"])
    rows = rows_from(g["nn"], g["flat"])
    tab, sx, sy, cut, n = ewald_golden()
    N = len(pos)
    F, C = O.split_generalized(g["genF"], N)
    u, D = O.real_space(pos, F, C, L, xy, rows, tab, sx, sy, cut, n)
    assert rel(u, g["real_vel"][:, :3]) < 2e-6
    # reference layout: delu[0] = (xx, xy, xz, yz), delu[1] = (yy, yx, zx, zy)
    d = g["real_delu"]
    ref = np.stack([d[:, 0], d[:, 1], d[:, 2], d[:, 5], d[:, 4], d[:, 3], d[:, 6], d[:, 7], d[:, 4] * 0], 1)
    got = np.stack([D[:, 0, 0], D[:, 0, 1], D[:, 0, 2], D[:, 1, 0], D[:, 1, 1], D[:, 1, 2], D[:, 2, 0], D[:, 2, 1],
                    D[:, 1, 1] * 0], 1)
    assert rel(got, ref) < 2e-6
    # couplet construction (TS2C) equals the oracle's
    c8 = g["couplet"]
    Cref = np.stack([c8[:, 0], c8[:, 1], c8[:, 2], c8[:, 5], c8[:, 4], c8[:, 3], c8[:, 6], c8[:, 7]], 1)
    Cgot = np.stack([C[:, 0, 0], C[:, 0, 1], C[:, 0, 2], C[:, 1, 0], C[:, 1, 1], C[:, 1, 2], C[:, 2, 0], C[:, 2, 1]], 1)
    assert rel(Cgot, Cref) < 1e-7


@pytest.mark.parametrize("case", ["green_even.npz", "green_mixed_sheared.npz"])
def test_green_oracle_matches_reference(case):
    g = golden(case)
    Nxyz = tuple(int(v) for v in g["Nxyz"])
    kx, ky, kz, w = O.gridk(Nxyz, tuple(g["L"]), float(g["xy"]), 0.5, float(g["eta"]))
    gk = g["gridk"].reshape(*Nxyz, 4)
    assert rel(kx, gk[..., 0]) < 1e-6 and rel(ky, gk[..., 1]) < 1e-6 and rel(w, gk[..., 3]) < 1e-6
    spec = g["spec_in"].astype(np.complex128).reshape(11, *Nxyz)
    Fh = spec[:3]
    order = [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2), (2, 0), (2, 1)]
    Ch = np.zeros((3, 3, *Nxyz), complex)
    for k, (a, b) in enumerate(order):
        Ch[a, b] = spec[3 + k]
    Ch[2, 2] = -(Ch[0, 0] + Ch[1, 1])
    U, D = O.green(Fh, Ch, gk[..., 0].astype(np.float64), gk[..., 1].astype(np.float64),
                   gk[..., 2].astype(np.float64), gk[..., 3].astype(np.float64))
    out = g["spec_out"].reshape(11, *Nxyz)
    assert rel(U, out[:3]) < 2e-6
    Dg = np.stack([D[a, b] for a, b in order])
    assert rel(Dg, out[3:]) < 2e-6


def test_precond_assembly_and_rcm_match_reference():
    g = golden("pairs_dense_sheared.npz")
    p = golden("precond_dense_sheared.npz")
    pos, L, xy = g["pos"], tuple(g["L"]), float(g["xy"])
    rows = rows_from(g["nn"], g["flat"])
    td, tv = O.resistance_table()
    A, prow = O.pruned_rfu_dense(pos, L, xy, rows, td, tv, relaxer=0.0)
    N = len(pos)
    ref = np.zeros((6 * N, 6 * N))
    np.add.at(ref, (p["coo_row"], p["coo_col"]), p["coo_val"].astype(np.float64))
    assert rel(A, ref) < 2e-6
    for a, b in zip(prow, rows_from(p["pn"], p["pflat"])):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    assert np.array_equal(O.rcm(prow), p["rcm_perm"])


def test_pair_force_and_strain_rhs_match_reference():
    g = golden("pairs_dense_sheared.npz")
    pos, L, xy = g["pos"], tuple(g["L"]), float(g["xy"])
    rows = rows_from(g["nn"], g["flat"])
    assert rel(O.pair_force(pos, L, xy, rows, T_ext=0.7), g["force"]) < 2e-6
    N = len(pos)
    got = O.strain_rhs(float(g["shear_rate"]), N, g["ori"], g["b2mask"], float(g["B2"]))
    assert rel(got, g["strain_rhs"]) < 1e-6


def test_euler_shear_matches_reference():
    g = golden("motion.npz")
    N = len(g["pos"])
    p, o, gb, img = O.euler_shear(g["pos"], g["ori"], g["gb"], g["vel"], np.zeros((N, 3), np.int64), tuple(g["L"]),
                                  float(g["xy"]), float(g["dt"]), float(g["shear_rate"]), float(g["B1"]),
                                  g["b1mask"], g["noise"])
    assert np.abs(p - g["pos_out"][:, :3]).max() < 1e-5
    assert np.abs(o - g["ori_out"]).max() < 1e-5
    assert np.abs(gb[:, :3] - g["gb_out"][:, :3]).max() < 1e-5
    assert np.array_equal(img, g["img_out"])


@pytest.mark.skipif(not R.available(), reason="reference harness not built here")
def test_oracle_matches_live_reference_random():
    from fsd_b200.configs import suspension
    rng = np.random.default_rng(5)
    for seed, phi, xy in [(1, 0.3, 0.1), (2, 0.5, -0.4)]:
        pos, Lc = suspension(120, phi, seed)
        L = (Lc, Lc, Lc)
        tab, sx, sy, cut, n = R.ewald_table(0.5, 1e-3)
        rows = O.neighbor_list(pos[:, :3], L, xy, cut + 0.4)
        td, tv = O.resistance_table()
        U6 = rng.standard_normal(6 * 120).astype(np.float32)
        assert rel(O.rfu(pos, U6, L, xy, rows, td, tv), R.rfu(pos, U6, rows, L, xy, td, tv)) < 2e-6
        assert rel(O.rsu(pos, U6, L, xy, rows, td, tv), R.rsu(pos, U6, rows, L, xy, td, tv)) < 2e-6
