"""Parity at the benchmarked suspension itself: N = 32768 unit spheres at
phi = 0.4 (seed 1, L = 70.01, 72^3 grid, P = 6), the configuration bench.py
times.  At this density the lubrication sub-list, the pruned contact graph
(about 4 blocks per row) and the two-hop sets (capped at 32) are as dense as
they get on the timed path, so each operator is checked here against the FP64
oracle on the same positions:

* mobility M^ff (wave + real space): 5e-5 relative (FP32 FFT against FP64);
* R_FU: 1e-5;
* saddle operator: 5e-5;
* the two-hop sparse approximate inverse G of the learned preconditioner,
  applied once, on a vector carried by 256 sampled particles: 1e-5 (the oracle
  solves only those columns; solving all 32768 in NumPy takes over 20 minutes).

The oracle's neighbour rows come from a k-d tree (same sorted rows as its
all-pairs list, which is slow at this size).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import ewald_golden
from fsd_b200.configs import suspension
from fsd_b200.core import FSD
from oracle import fsd_oracle as O

pytestmark = pytest.mark.gpu

N, PHI, SEED = 32768, 0.4, 1
TOL_PAIR = 1e-5
TOL_WAVE = 5e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x, np.float32)).cuda().contiguous().view(-1)


@pytest.fixture(scope="module")
def bench_case(cuda):
    pos, Lc = suspension(N, PHI, seed=SEED)
    L = (Lc, Lc, Lc)
    table = ewald_golden()
    rows = O.neighbor_list_kdtree(pos, L, table[3] + 0.4)
    pr = O.Problem(pos, L, 0.0, table=table, rows=rows)
    return pos, Lc, pr


def test_grid_is_the_benchmarked_one(bench_case):
    pos, Lc, pr = bench_case
    assert (pr.gp["Nx"], pr.gp["Ny"], pr.gp["Nz"], pr.gp["P"]) == (72, 72, 72, 6)


def test_mobility_at_bench_config(bench_case):
    pos, Lc, pr = bench_case
    s = FSD(N, (Lc, Lc, Lc, 0.0))
    p = dev(pos)
    s.build_neighbor_list(p)
    F = np.random.default_rng(21).standard_normal(11 * N)
    assert rel(s.mobility(p, dev(F)).cpu().numpy(), pr.mobility(F)) < TOL_WAVE
    s.close()


def test_rfu_at_bench_config(bench_case):
    pos, Lc, pr = bench_case
    s = FSD(N, (Lc, Lc, Lc, 0.0))
    p = dev(pos)
    s.build_neighbor_list(p)
    U = np.random.default_rng(22).standard_normal(6 * N)
    assert rel(s.rfu(p, dev(U)).cpu().numpy(), pr.rfu(U)) < TOL_PAIR
    s.close()


def test_saddle_multiply_at_bench_config(bench_case):
    pos, Lc, pr = bench_case
    s = FSD(N, (Lc, Lc, Lc, 0.0))
    p = dev(pos)
    s.build_neighbor_list(p)
    x = np.random.default_rng(23).standard_normal(17 * N)
    assert rel(s.saddle_multiply(p, dev(x)).cpu().numpy(), pr.saddle_multiply(x)) < TOL_WAVE
    s.close()


def test_two_hop_approximate_inverse_at_bench_config(bench_case):
    pos, Lc, pr = bench_case
    s = FSD(N, (Lc, Lc, Lc, 0.0), precond="learned", learned_inner=0)
    p = dev(pos)
    s.build_neighbor_list(p)
    s.precond_build(p)
    rng = np.random.default_rng(24)
    cols = np.sort(rng.choice(N, 256, replace=False))
    v = np.zeros((N, 6))
    v[cols] = rng.standard_normal((len(cols), 6))
    # saddle preconditioner input whose lubrication part is t = v: then x[11N:] = G v
    b = np.zeros(17 * N)
    b[11 * N:] = -v.ravel()
    got = s.precond_apply(dev(b)).cpu().numpy()[11 * N:].reshape(N, 6)
    A = O.pruned_rfu_sparse(pr.pos, pr.L, 0.0, pr.tdist, pr.tvals, rows=pr.rows, rp=pr.rp).tocsr()
    blocks = O.spai2_columns(A, N, [int(c) for c in cols])
    ref = np.zeros((N, 6))
    for (srow, c), X in blocks.items():
        ref[srow] += X @ v[c]
    assert rel(got, ref) < TOL_PAIR
    s.close()
