"""Checkpoint and resume of the solver state a step carries (the carried
state of Stokes::integrateStepOne, Stokes.cc:1658-1666, and the main solve's
warm start, Integrator.cu:777).

* A checkpoint of another size or with a damaged header is refused with
  FSD_ERR_BAD_PARAMS, not read.
* Three Brownian steps with shear on one handle; the same first two on a
  second handle, whose checkpoint and caller arrays (positions,
  orientations, images) then resume a third, fresh handle: its third step
  equals the first handle's bit for bit, with IChol (whose relaxer is part
  of the carried state) and with the learned preconditioner.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from fsd_b200 import _lib
from fsd_b200.configs import suspension
from fsd_b200.core import FSD


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["ichol", "learned"])
def test_resume_from_checkpoint_continues_bit_for_bit(cuda, precond):
    N = 400
    pos, Lc = suspension(N, 0.3, 12)
    kw = dict(T=1.0, dt=1e-4, seed=21, solver_tol=1e-4, precond=precond, period=1)

    def state():
        return (torch.as_tensor(pos).cuda().view(-1).contiguous(),
                torch.tensor([0.0, 0.0, 1.0], device="cuda").repeat(N),
                torch.zeros(3 * N, dtype=torch.int32, device="cuda"),
                torch.zeros(6 * N, device="cuda"), torch.zeros(11 * N, device="cuda"))

    a = FSD(N, (Lc, Lc, Lc, 0.1), **kw)
    p, o, im, F, V = state()
    for t in range(3):
        a.step(t, 0.5, p, o, im, F, V, raise_on_error=False)
    ref = (p.cpu().numpy(), o.cpu().numpy(), im.cpu().numpy(), V.cpu().numpy())
    a.close()
    b = FSD(N, (Lc, Lc, Lc, 0.1), **kw)
    p, o, im, F, V = state()
    for t in range(2):
        b.step(t, 0.5, p, o, im, F, V, raise_on_error=False)
    ck = b.checkpoint()
    b.close()
    c = FSD(N, (Lc, Lc, Lc, 0.1), **kw)
    c.restore(ck)
    c.step(2, 0.5, p, o, im, F, V, raise_on_error=False)
    got = (p.cpu().numpy(), o.cpu().numpy(), im.cpu().numpy(), V.cpu().numpy())
    c.close()
    for x, y in zip(got, ref):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_checkpoint_of_another_size_is_refused(cuda):
    s = FSD(100, (20.0, 20.0, 20.0, 0.0))
    ck = bytearray(s.checkpoint())
    assert len(ck) == _lib.lib().fsd_checkpoint_size(s._h)
    other = FSD(120, (20.0, 20.0, 20.0, 0.0))
    buf = C.create_string_buffer(bytes(ck), len(ck))
    assert _lib.lib().fsd_checkpoint_load(other._h, buf, len(ck)) == 1  # FSD_ERR_BAD_PARAMS
    ck[0] ^= 0xFF  # damaged header
    buf = C.create_string_buffer(bytes(ck), len(ck))
    assert _lib.lib().fsd_checkpoint_load(s._h, buf, len(ck)) == 1
    s.close()
    other.close()
