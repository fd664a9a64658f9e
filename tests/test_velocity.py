"""Velocities and stresslets of one velocity computation (fsd_compute_velocity,
Integrator_ComputeVelocity at kT = 0) against the FP64 oracle: the dilute
suspension of N = 1000 at phi = 0.2 without shear, and a sheared, tilted
dense case.
GMRES runs to 1e-6 (5e-7 for the dense sheared case, whose small relative
velocities amplify the solver's residual: 1e-6 leaves 1.005e-4 there, 5e-7
leaves 4.5e-5) so that solver error stays under the 1e-4 bar on velocities
and stresslets (relative 2-norm); the FP32 residual floor near 2e-7 keeps
the tolerance above that.  The interparticle force must agree to 1e-5."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import ewald_golden
from fsd_b200.configs import suspension
from fsd_b200.core import FSD
from oracle import fsd_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.mark.parametrize("N,phi,seed,shear,xy,precond,tol", [(1000, 0.2, 1, 0.0, 0.0, "ichol", 1e-6),
                                                               (1000, 0.2, 1, 0.0, 0.0, "learned", 1e-6),
                                                               (400, 0.35, 2, 1.0, 0.15, "learned", 5e-7)])
def test_velocity_and_stresslet_match_oracle(cuda, N, phi, seed, shear, xy, precond, tol):
    pos, Lc = suspension(N, phi, seed)
    L = (Lc, Lc, Lc)
    s = FSD(N, (Lc, Lc, Lc, xy), T=0.0, dt=1e-4, period=1, solver_tol=tol, precond=precond,
            gmres_max_iter=4000)
    p = torch.as_tensor(pos, device="cuda").view(-1).contiguous()
    ori = torch.as_tensor(np.tile([0.0, 0.0, 1.0], N).astype(np.float32), device="cuda")
    img = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
    F = torch.zeros(6 * N, device="cuda")
    V = torch.zeros(11 * N, device="cuda")
    s.compute_velocity(0, shear, p, ori, img, F, V)
    v = V.cpu().numpy().astype(np.float64)
    pr = O.Problem(pos, L, xy, table=ewald_golden())
    U, S, Fo = pr.velocity(shear)
    assert rel(F.cpu().numpy(), Fo) < 1e-5
    assert rel(v[:6 * N], U) < 1e-4
    assert rel(v[6 * N:], S) < 1e-4
    s.close()
