"""The seeded synthetic suspensions (random sequential addition, then
overlap relaxation): every configuration the tests and the benchmark use
holds the minimum surface gap of 1e-3, including dense boxes above random
sequential addition's jamming fraction, where a second relaxation phase
(pushes toward three times the gap) removes the overlaps the first phase
leaves; the same seed gives the same positions."""
from __future__ import annotations

import numpy as np
import pytest

from fsd_b200.configs import box_length, min_gap, suspension


@pytest.mark.parametrize("phi", [0.2, 0.4, 0.55])
def test_suspension_holds_the_minimum_gap(phi):
    N = 2000
    pos, L = suspension(N, phi, seed=7)
    assert pos.shape == (N, 4) and pos.dtype == np.float32
    assert abs(L - box_length(N, phi)) < 1e-12
    assert np.all(pos[:, :3] >= -L / 2) and np.all(pos[:, :3] < L / 2)
    assert min_gap(pos, L) > 1e-3 - 2e-5  # float32 storage of coordinates near L/2


def test_suspension_is_reproducible():
    a, _ = suspension(500, 0.3, seed=3)
    b, _ = suspension(500, 0.3, seed=3)
    c, _ = suspension(500, 0.3, seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_cpu_full_step_runs_to_convergence():
    """The host-core baseline's complete FP64 step (oracle.cpu_step) on a small
    box: every solve converges within its restart and the stage times add up."""
    from conftest import ewald_golden
    from oracle.cpu_step import full_step_seconds
    pos, L = suspension(200, 0.3, seed=2)
    sec, parts, its = full_step_seconds(pos, L, ewald_golden())
    assert sec > 0 and sum(parts.values()) <= sec * 1.01
    assert 0 < its["gmres_main"] < 200 and 0 < its["gmres_rfd_plus"] < 200
    assert its["lanczos_ff"] >= 2 and its["lanczos_nf"] >= 2


def test_smoothed_interval_target_avoids_a_cliff():
    """The interval-network training target with --smooth: the candidate whose
    iteration count, averaged in log with its neighbours, is lowest -- so a
    lone minimum next to a steep rise loses to a flat valley."""
    from fsd_b200.train_precond import smoothed_best
    its = {0.01: 900, 0.02: 60, 0.03: 400, 0.045: 80, 0.07: 78, 0.1: 82, 0.15: 120}
    assert min(its, key=its.get) == 0.02
    assert smoothed_best(its) == 0.07
    its[0.03] = 10 ** 9  # a candidate that never converged counts as infinitely bad
    assert smoothed_best(its) == 0.07


def test_configuration_cache_round_trip(tmp_path):
    from fsd_b200.train_precond import configuration
    a, La = configuration(300, 0.3, 5, tmp_path)
    assert (tmp_path / "susp_N300_phi0.3_s5.npz").exists()
    b, Lb = configuration(300, 0.3, 5, tmp_path)
    c, _ = suspension(300, 0.3, seed=5)
    assert La == Lb and np.array_equal(a, b) and np.array_equal(a, c)


def test_cpu_lanczos_square_root_matches_dense():
    """The Chow-Saad Lanczos square root of the host-core baseline against a
    dense eigendecomposition, on a small SPD matrix with the spread of
    eigenvalues of a lubrication block (1e-3 to 1)."""
    from oracle.cpu_step import _lanczos_sqrt
    rng = np.random.default_rng(4)
    n = 60
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.geomspace(1e-3, 1.0, n)
    A = (Q * ev) @ Q.T
    z = rng.standard_normal(n)
    y, m = _lanczos_sqrt(lambda v: A @ v, z, tol=1e-10, max_iter=n)
    ref = (Q * np.sqrt(ev)) @ (Q.T @ z)
    assert np.linalg.norm(y - ref) < 1e-6 * np.linalg.norm(ref)
    assert m <= n
