"""CUDA path through the C ABI against the oracle and the reference's golden outputs.

Tolerances: the CUDA path computes in FP32 (as the reference does); results
are compared in relative 2-norm against FP64 restatements.  Pair sums and table
interpolation agree to ~1e-6; wave-space results (FP32 FFT vs FP64 FFT) to
~1e-5.  The bar is 1e-4 relative in velocities.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import ewald_golden, golden, rows_from
from fsd_b200.configs import suspension
from fsd_b200.core import FSD
from oracle import fsd_oracle as O

pytestmark = pytest.mark.gpu

TOL_PAIR = 1e-5
TOL_WAVE = 5e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x, np.float32)).cuda().contiguous().view(-1)


def solver_for(pos, L, xy=0.0, **kw):
    N = len(pos)
    s = FSD(N, (L[0], L[1], L[2], xy), **kw)
    p = dev(pos).view(N, 4).contiguous()
    s.build_neighbor_list(p.view(-1))
    return s, p.view(-1)


def problem(pos, L, xy=0.0):
    return O.Problem(pos, L, xy, table=ewald_golden())


@pytest.mark.parametrize("case", ["pairs_dilute.npz", "pairs_dense_sheared.npz"])
def test_neighbor_list_equals_brute_force(cuda, case):
    g = golden(case)
    L, xy = tuple(g["L"]), float(g["xy"])
    s, p = solver_for(g["pos"], L, xy)
    got = s.neighbor_list()
    ref = O.neighbor_list(g["pos"], L, xy, s.pse_info().ewald_cut + 0.4)
    for a, b in zip(got, ref):
        assert np.array_equal(np.sort(a), b)


def test_neighbor_list_large_cell_path(cuda):
    pos, Lc = suspension(3000, 0.35, 3)
    L = (Lc, Lc, Lc)
    s, p = solver_for(pos, L, 0.2)
    got = s.neighbor_list()
    ref = O.neighbor_list(pos, L, 0.2, s.pse_info().ewald_cut + 0.4)
    assert all(np.array_equal(np.sort(a), b) for a, b in zip(got, ref))


@pytest.mark.parametrize("case", ["pairs_dilute.npz", "pairs_dense_sheared.npz"])
def test_lubrication_equals_reference(cuda, case):
    g = golden(case)
    L, xy = tuple(g["L"]), float(g["xy"])
    s, p = solver_for(g["pos"], L, xy)
    U = dev(g["U6"])
    ori, mask, B2, sr = dev(g["ori"]), dev(g["b2mask"]), float(g["B2"]), float(g["shear_rate"])
    assert rel(s.rfu(p, U).cpu(), g["rfu"]) < TOL_PAIR
    assert rel(s.rfe(p, sr, ori, mask, B2).cpu(), g["rfe"]) < TOL_PAIR
    assert rel(s.rsu(p, U).cpu(), g["rsu"]) < TOL_PAIR
    assert rel(s.rse(p, sr, ori, mask, B2).cpu(), g["rse"]) < TOL_PAIR


@pytest.mark.parametrize("case", ["pairs_dilute.npz", "pairs_dense_sheared.npz"])
def test_real_space_mobility(cuda, case):
    g = golden(case)
    L, xy = tuple(g["L"]), float(g["xy"])
    s, p = solver_for(g["pos"], L, xy)
    pr = problem(g["pos"], L, xy)
    got = s.mobility(p, dev(g["genF"]), parts=2).cpu().numpy()
    assert rel(got, pr.mobility(g["genF"], parts=2)) < TOL_PAIR


@pytest.mark.parametrize("case", ["pairs_dilute.npz", "pairs_dense_sheared.npz"])
def test_wave_space_mobility(cuda, case):
    g = golden(case)
    L, xy = tuple(g["L"]), float(g["xy"])
    s, p = solver_for(g["pos"], L, xy)
    pr = problem(g["pos"], L, xy)
    got = s.mobility(p, dev(g["genF"]), parts=1).cpu().numpy()
    assert rel(got, pr.mobility(g["genF"], parts=1)) < TOL_WAVE


@pytest.mark.parametrize("N,phi,xy,seed", [(1000, 0.2, 0.0, 1), (400, 0.35, 0.45, 2), (8192, 0.1, 0.0, 3),
                                            (1024, 0.1, 0.3, 4), (8000, 0.1, 0.2, 5)])
def test_full_mobility(cuda, N, phi, xy, seed):
    """Grids 27^3, 18^3, 72^3, 36^3 and a tilted 72^3: the y and z FFT passes run
    as one plane kernel for 27, 36 and 72 and as separate line passes for 18;
    spreading uses tile-relative separations on the two 72^3 grids and the
    per-node minimum image on the others."""
    pos, Lc = suspension(N, phi, seed)
    L = (Lc, Lc, Lc)
    s, p = solver_for(pos, L, xy)
    pr = problem(pos, L, xy)
    F = np.random.default_rng(seed).standard_normal(11 * N)
    got = s.mobility(p, dev(F)).cpu().numpy()
    assert rel(got, pr.mobility(F)) < TOL_WAVE


def test_mobility_is_symmetric_positive(cuda):
    pos, Lc = suspension(30, 0.1, 4)
    L = (Lc, Lc, Lc)
    s, p = solver_for(pos, L, 0.1)
    n = 11 * 30
    M = np.stack([s.mobility(p, dev(np.eye(n)[k])).cpu().numpy() for k in range(n)], 1)
    assert np.abs(M - M.T).max() < 2e-5 * np.abs(M).max()
    assert np.linalg.eigvalsh(0.5 * (M + M.T)).min() > 0


def test_saddle_multiply(cuda):
    g = golden("pairs_dense_sheared.npz")
    L, xy = tuple(g["L"]), float(g["xy"])
    s, p = solver_for(g["pos"], L, xy)
    pr = problem(g["pos"], L, xy)
    x = np.random.default_rng(7).standard_normal(17 * len(g["pos"]))
    assert rel(s.saddle_multiply(p, dev(x)).cpu().numpy(), pr.saddle_multiply(x)) < TOL_WAVE


def test_preconditioner_equals_ichol_of_reference_ordering(cuda):
    g = golden("pairs_dense_sheared.npz")
    pc = golden("precond_dense_sheared.npz")
    L, xy = tuple(g["L"]), float(g["xy"])
    N = len(g["pos"])
    s, p = solver_for(g["pos"], L, xy, precond="ichol", ichol_local_shift=0)
    s.precond_build(p)
    relaxer = s.solve_info()["ichol_relaxer"]
    td, tv = O.resistance_table()
    A, prow = O.pruned_rfu_dense(g["pos"], L, xy, rows_from(g["nn"], g["flat"]), td, tv, relaxer=relaxer)
    perm = pc["rcm_perm"]
    P6 = (6 * perm[:, None] + np.arange(6)).ravel()
    B = A[np.ix_(P6, P6)]
    pattern = np.zeros((N, N), bool)
    inv = np.argsort(perm)
    for i, r in enumerate(prow):
        pattern[inv[i], inv[np.asarray(r)]] = True
    Lf = O.ichol0_dense(B, np.kron(pattern, np.ones((6, 6), bool)))
    assert Lf is not None
    Gp = np.linalg.inv(Lf @ Lf.T)
    G = np.zeros_like(Gp)
    G[np.ix_(P6, P6)] = Gp
    b = np.random.default_rng(8).standard_normal(17 * N)
    got = s.precond_apply(dev(b)).cpu().numpy()
    assert rel(got, O.saddle_precond(b, G, N)) < 1e-4


@pytest.mark.parametrize("precond,restart,inner", [("ichol", 100, 0), ("none", 100, 0), ("ichol", 7, 0),
                                                  ("learned", 7, 0), ("learned", 7, 3)])
def test_saddle_solve_matches_dense_solution(cuda, precond, restart, inner):
    """Restart 7 runs several GMRES cycles: with a fixed preconditioner the
    solution is mapped back through the delayed re-orthogonalisation's
    coefficients, with inner steps (flexible GMRES) through the kept Z basis."""
    N = 80
    pos, Lc = suspension(N, 0.2, 9)
    L = (Lc, Lc, Lc)
    s, p = solver_for(pos, L, 0.0, precond=precond, solver_tol=1e-6, gmres_restart=restart, learned_inner=inner)
    s.precond_build(p)
    pr = problem(pos, L)
    rhs = np.random.default_rng(10).standard_normal(17 * N)
    x, it, res, st = s.saddle_solve(p, dev(rhs))
    ref = pr.solve(rhs)
    assert res < 1e-5
    assert rel(x.cpu().numpy(), ref) < 1e-4
    assert rel(x.cpu().numpy()[11 * N:], ref[11 * N:]) < 1e-4


def test_step_deterministic_and_finite(cuda):
    N = 300
    pos, Lc = suspension(N, 0.3, 12)
    s = FSD(N, (Lc, Lc, Lc, 0.0), T=1.0, dt=1e-4, seed=5, solver_tol=1e-4, period=1)
    outs = []
    for rep in range(2):
        s2 = FSD(N, (Lc, Lc, Lc, 0.0), T=1.0, dt=1e-4, seed=5, solver_tol=1e-4, period=1)
        p = dev(pos)
        ori = dev(np.tile([0.0, 0.0, 1.0], N))
        img = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
        F = torch.zeros(6 * N, device="cuda")
        V = torch.zeros(11 * N, device="cuda")
        for t in range(3):
            s2.step(t, 0.5, p, ori, img, F, V)
        torch.cuda.synchronize()
        outs.append((p.cpu().numpy().copy(), V.cpu().numpy().copy()))
        info = s2.solve_info()
        assert info["gmres_resid"][2] < 1e-4
        s2.close()
    assert np.isfinite(outs[0][0]).all() and np.isfinite(outs[0][1]).all()
    assert np.array_equal(outs[0][0], outs[1][0]), "same seed must reproduce the trajectory bit for bit"
    moved = np.abs(outs[0][0] - pos.ravel()).max()
    assert 0 < moved < 1.0
    s.close()


def test_autotuned_shapes_give_the_same_mobility(cuda):
    """The autotuner only changes launch shapes (spreading tile, FFT batches),
    so the mobility agrees with the fixed shapes to rounding."""
    pos, Lc = suspension(2000, 0.3, 8)
    L = (Lc, Lc, Lc)
    F = dev(np.random.default_rng(8).standard_normal(11 * 2000))
    out = []
    for tune in (0, 1):
        s, p = solver_for(pos, L, 0.1, autotune=tune)
        out.append(s.mobility(p, F).cpu().numpy())
        s.close()
    assert rel(out[1], out[0]) < 1e-6
