"""The learned inner polynomial of FSD_PRECOND_LEARNED (learned_poly mode):
y = G q(AG) t with a Chebyshev polynomial q whose coefficients the
message-passing network predicts per configuration, against the FP64 oracle
(oracle/mpnn_oracle.py).

* Application: the library's Clenshaw recurrence (2k - 1 SpMV kernels) against
  the FP64 recurrence with the same coefficients and spectral bound: 1e-5
  relative (FP32 products of G and A).
* Training signal: the network's coefficients (mean over particles of its node
  head), the loss E_t ||t - AG q(AG) t||^2 / ||t||^2 on the library's probe
  draws, and the weight gradient along random directions against central
  differences of the FP64 oracle loss: coefficients 1e-5, loss 1e-4, gradient
  5e-3 with the FP32 layers (the FP32 backward through three message-passing
  layers measured 3e-3); 3e-2 / 3e-2 / 6e-2 with the BF16 tensor-core layers.  The least-squares optimum it reports must not be above the loss.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from fsd_b200.configs import suspension
from fsd_b200.core import FSD
from oracle import mpnn_oracle as M

pytestmark = pytest.mark.gpu

K = 8


def _setup(N=300, phi=0.4, seed=4, **kw):
    pos, Lc = suspension(N, phi, seed)
    s = FSD(N, (Lc, Lc, Lc, 0.0), precond="learned", learned_poly=K, **kw)
    p = torch.as_tensor(pos).cuda().view(-1).contiguous()
    s.build_neighbor_list(p)
    return s, p, M.problem(pos, (Lc, Lc, Lc), 0.0)


def test_polynomial_application_matches_oracle(cuda):
    s, p, pr = _setup()
    c = np.array([1.4, -0.9, 0.5, -0.3, 0.17, -0.09, 0.05, -0.02], np.float32)
    s.learned_set_poly(c)
    s.precond_build(p)
    cg, lam = s.learned_get_poly()
    assert np.array_equal(cg, c) and 1.0 < lam < 3.0
    N = pr["N"]
    b = np.random.default_rng(2).standard_normal(17 * N)
    got = s.precond_apply(torch.as_tensor(b, dtype=torch.float32).cuda()).cpu().numpy()
    ref = M.poly_apply(b.astype(np.float32).astype(np.float64), c.astype(np.float64), np.float64(np.float32(lam)),
                       pr["A"], pr["G0"], N)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5
    s.close()


@pytest.mark.parametrize("tensor_cores,tol_c,tol_l,tol_g", [(False, 1e-5, 1e-4, 5e-3), (True, 3e-2, 3e-2, 6e-2)])
def test_poly_loss_and_gradient_match_oracle(cuda, tensor_cores, tol_c, tol_l, tol_g):
    s, p, pr = _setup()
    s.learned_tensor_cores(tensor_cores)
    w = M.init_weights(0, head_scale=0.05)
    s.learned_set_weights(w)
    P, step = 3, 5
    out = s.learned_poly_train_step(p, n_probes=P, step=step, want_grad=True)
    _, lam = s.learned_get_poly()
    N = pr["N"]
    T = s.draw_normals(7, step, P * 6 * N).cpu().numpy().astype(np.float64).reshape(P, 6 * N)
    wd = w.astype(np.float64)
    lam = float(np.float32(lam))
    c_ref = M.poly_coeffs(wd, pr, K)
    assert np.linalg.norm(out["coef"] - c_ref) <= tol_c * np.linalg.norm(c_ref)
    ref = M.poly_loss(wd, pr, T, lam, K)
    assert abs(out["loss"] - ref) <= tol_l * abs(ref)
    assert out["loss_opt"] <= out["loss"] * (1 + 1e-4)
    rng = np.random.default_rng(1)
    for _ in range(3):
        d = rng.standard_normal(len(w))
        eps = 1e-4
        fd = (M.poly_loss(wd + eps * d, pr, T, lam, K) - M.poly_loss(wd - eps * d, pr, T, lam, K)) / (2 * eps)
        assert abs(float(out["grad"].astype(np.float64) @ d) - fd) <= tol_g * abs(fd)
    s.close()
