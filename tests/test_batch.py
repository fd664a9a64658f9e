"""Batched stepping of independent suspensions (fsd_step_batch): replicas of
uneven size stepped concurrently on their own streams give bit for bit the
trajectories of stepping them one by one."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from fsd_b200.configs import suspension
from fsd_b200.core import FSD, step_batch

pytestmark = pytest.mark.gpu

CASES = [(300, 0.25, 1, 0.5), (520, 0.35, 2, 1.0), (400, 0.15, 3, 0.0)]


def _replicas():
    reps = []
    for N, phi, seed, rate in CASES:
        pos, L = suspension(N, phi, seed)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            s = FSD(N, (L, L, L, 0.0), T=1.0, dt=1e-4, seed=seed, solver_tol=1e-4, precond="learned",
                    learned_inner=4, gmres_restart=60)
            st = dict(p=torch.as_tensor(pos, device="cuda").view(-1).contiguous(),
                      ori=torch.as_tensor(np.tile([0.0, 0.0, 1.0], N).astype(np.float32), device="cuda"),
                      img=torch.zeros(3 * N, dtype=torch.int32, device="cuda"),
                      F=torch.zeros(6 * N, device="cuda"), V=torch.zeros(11 * N, device="cuda"))
        torch.cuda.synchronize()
        reps.append((s, st, rate, stream))
    return reps


def test_batched_steps_equal_sequential_steps(cuda):
    seq = _replicas()
    for t in range(2):
        for s, st, rate, stream in seq:
            with torch.cuda.stream(stream):
                s.step(t, rate, st["p"], st["ori"], st["img"], st["F"], st["V"])
    torch.cuda.synchronize()
    bat = _replicas()
    for t in range(2):
        args = [s.step_args(t, rate, st["p"], st["ori"], st["img"], st["F"], st["V"]) for s, st, rate, _ in bat]
        status = step_batch([r[0] for r in bat], args)
        assert all(x in (0, 4) for x in status)
    torch.cuda.synchronize()
    for (s1, a, _, _), (s2, b, _, _) in zip(seq, bat):
        assert torch.equal(a["p"], b["p"]) and torch.equal(a["V"], b["V"])
        assert np.isfinite(b["p"].cpu().numpy()).all()
        s1.close()
        s2.close()
