"""Brownian terms: statistics against the FP64 oracle's mobility and resistance.

The reference draws its normals from cuRAND (closed), so parity is
statistical: the far-field slip U = sqrt(2kT/dt) M^1/2 psi
(Brownian_FarField.cu:829-1061, wave-space random field plus Lanczos on the
real-space part) must have covariance 2kT/dt M, and the near-field force
F = sqrt(2kT/dt) R_FU^1/2 psi (Brownian_NearField.cu:407-464) covariance
2kT/dt R_FU.  They are checked along fixed random directions v: the sample
variance of v.U over S draws has relative standard error sqrt(2/S) (S = 3000:
2.6%), so the bar is 10%; sample covariances of direction pairs must match to
0.1 of sqrt(var1 var2); means must vanish to 4 standard errors.
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

N, PHI, SEED, S, NDIR = 80, 0.2, 21, 3000, 6


def _system(T=1.0, dt=1.0):
    pos, Lc = suspension(N, PHI, SEED)
    L = (Lc, Lc, Lc)
    s = FSD(N, (Lc, Lc, Lc, 0.0), T=T, dt=dt, seed=7, lanczos_tol=1e-4, lanczos_max=100)
    p = torch.as_tensor(pos).cuda().view(-1).contiguous()
    s.build_neighbor_list(p)
    return s, p, pos, L


def _check(samples, dirs, C_dirs, scale):
    """samples (S, n); dirs (m, n); C_dirs[a][b] = v_a^T C v_b of the target covariance."""
    proj = samples @ dirs.T                       # (S, m)
    mean = proj.mean(0)
    cov = np.cov(proj.T)
    target = scale * C_dirs
    var = np.diag(target)
    assert np.all(np.abs(mean) < 4 * np.sqrt(var / len(samples)))
    assert np.all(np.abs(np.diag(cov) - var) < 0.10 * var)
    off = np.abs(cov - target) / np.sqrt(np.outer(var, var))
    assert off.max() < 0.10


def test_farfield_slip_covariance_is_2kT_over_dt_times_mobility(cuda):
    s, p, pos, L = _system()
    samples = np.stack([s.brownian_farfield(p, t).cpu().numpy().astype(np.float64) for t in range(S)])
    pr = O.Problem(pos, L, table=ewald_golden())
    dirs = np.random.default_rng(3).standard_normal((NDIR, 11 * N))
    Mv = np.stack([pr.mobility(v) for v in dirs])
    _check(samples, dirs, dirs @ Mv.T, 2.0)
    info = s.solve_info()
    assert info["lanczos_ff_err"] < 1e-3
    s.close()


def test_nearfield_force_covariance_is_2kT_over_dt_times_rfu(cuda):
    s, p, pos, L = _system()
    samples = np.stack([s.brownian_nearfield(p, t).cpu().numpy().astype(np.float64) for t in range(S)])
    pr = O.Problem(pos, L, table=ewald_golden())
    dirs = np.random.default_rng(4).standard_normal((NDIR, 6 * N))
    Rv = np.stack([pr.rfu(v) for v in dirs])
    _check(samples, dirs, dirs @ Rv.T, 2.0)
    s.close()


def test_rfd_drift_is_linear_in_temperature_and_reproducible(cuda):
    pos, Lc = suspension(N, PHI, SEED)
    img = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
    out = []
    for T in (1.0, 2.0, 2.0):
        s = FSD(N, (Lc, Lc, Lc, 0.0), T=T, dt=1.0, seed=7, solver_tol=1e-6)
        p = torch.as_tensor(pos).cuda().view(-1).contiguous()
        s.build_neighbor_list(p)
        s.precond_build(p)
        out.append(s.rfd_drift(p, img, 5).cpu().numpy().astype(np.float64))
        s.close()
    assert np.isfinite(out[0]).all() and np.abs(out[0]).max() > 0
    assert np.array_equal(out[1], out[2])
    assert np.linalg.norm(out[1] - 2 * out[0]) <= 1e-3 * np.linalg.norm(out[1])
