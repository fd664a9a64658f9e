"""The learned Chebyshev interval of the inner polynomial (the default
learned_poly mode).

* The coefficients of the interval polynomial (fsd_learned_interval_coefficients,
  Chebyshev interpolation in FP64) against an FP64 least-squares restatement:
  1e-9 relative; and the residual polynomial 1 - x q(x) stays within [-1, 1]
  on [0, lambda] (no eigenvalue of AG amplified) and below the Chebyshev bound
  on [rho lambda, lambda].
* The interval network's training signal on the GPU: the predicted log rho
  (mean over particles of the node head's first output) and the gradient of
  the squared error against the FP64 oracle: prediction 1e-5, gradient
  along random directions 5e-3 (the FP32 backward through three
  message-passing layers measured 4e-3).
* A build with a fixed interval uses it (solve info) and its application
  matches the oracle's FP64 Clenshaw evaluation of the same coefficients:
  1e-4.  The interval polynomial's Chebyshev coefficients alternate in sign
  with sum of magnitudes near 45 (rho = 0.05, ten terms), so the recurrence
  amplifies FP32 rounding about 45-fold (2.5e-5 measured).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from fsd_b200 import _lib
from fsd_b200.configs import suspension
from fsd_b200.core import FSD
from oracle import mpnn_oracle as M


def _coeffs(rho, lam, k):
    c = np.zeros(k, np.float32)
    assert _lib.lib().fsd_learned_interval_coefficients(rho, lam, k, c.ctypes.data_as(C.c_void_p)) == 0
    return c


def _cheb_eval(c, u):
    return sum(cm * np.cos(m * np.arccos(2 * u - 1)) for m, cm in enumerate(c))


@pytest.mark.parametrize("rho,k", [(0.05, 10), (0.02, 8), (0.15, 12)])
def test_interval_coefficients_match_oracle_and_bound_the_residual(rho, k):
    lam = 1.37
    c = _coeffs(rho, lam, k).astype(np.float64)
    ref = M.interval_coefficients(rho, k) / lam
    assert np.linalg.norm(c - ref) <= 1e-6 * np.linalg.norm(ref)  # FP32 storage of the coefficients
    u = np.linspace(0.0, 1.0, 2001)
    r = 1.0 - u * lam * _cheb_eval(c, u)
    assert np.all(np.abs(r) <= 1.0 + 1e-4)
    zs = (1 + rho) / (1 - rho)
    bound = 1.0 / np.cosh(k * np.arccosh(zs))
    assert np.max(np.abs(r[u >= rho])) <= bound * (1 + 1e-3) + 1e-6


@pytest.mark.gpu
def test_ratio_prediction_and_gradient_match_oracle(cuda):
    N = 300
    pos, Lc = suspension(N, 0.4, 4)
    s = FSD(N, (Lc, Lc, Lc, 0.0), precond="learned", learned_poly=10)
    s.learned_tensor_cores(False)
    p = torch.as_tensor(pos).cuda().view(-1).contiguous()
    s.build_neighbor_list(p)
    pr = M.problem(pos, (Lc, Lc, Lc), 0.0)
    w = M.init_weights(0, head_scale=0.05)
    s.learned_set_weights(w)
    target = float(np.log(0.04))
    loss, pred = s.learned_ratio_train_step(p, target, lr=0.0)
    wd = w.astype(np.float64)
    _, on = M.forward(wd, pr["x"], pr["i"], pr["j"], pr["N"])
    assert abs(pred - on[:, 0].mean()) <= 1e-5 * max(1.0, abs(on[:, 0].mean()))
    assert abs(loss - M.ratio_loss(wd, pr, target)) <= 1e-4 * max(M.ratio_loss(wd, pr, target), 1e-6)
    _, _, g = s.learned_ratio_train_step(p, target, lr=0.0, want_grad=True)
    rng = np.random.default_rng(1)
    for _ in range(3):
        d = rng.standard_normal(len(w))
        eps = 1e-4
        fd = (M.ratio_loss(wd + eps * d, pr, target) - M.ratio_loss(wd - eps * d, pr, target)) / (2 * eps)
        assert abs(float(g.astype(np.float64) @ d) - fd) <= 5e-3 * abs(fd)
    s.close()


@pytest.mark.gpu
def test_fixed_interval_application_matches_oracle(cuda):
    N = 300
    pos, Lc = suspension(N, 0.4, 4)
    s = FSD(N, (Lc, Lc, Lc, 0.0), precond="learned", learned_poly=10, poly_interval=0.05)
    p = torch.as_tensor(pos).cuda().view(-1).contiguous()
    s.build_neighbor_list(p)
    s.precond_build(p)
    info = s.solve_info()
    assert info["poly_source"] == 4 and abs(info["poly_ratio"] - 0.05) < 1e-7
    c, lam = s.learned_get_poly()
    pr = M.problem(pos, (Lc, Lc, Lc), 0.0)
    b = np.random.default_rng(2).standard_normal(17 * N)
    got = s.precond_apply(torch.as_tensor(b, dtype=torch.float32).cuda()).cpu().numpy()
    ref = M.poly_apply(b.astype(np.float32).astype(np.float64), c.astype(np.float64), np.float64(np.float32(lam)),
                       pr["A"], pr["G0"], N)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-4
    s.close()
