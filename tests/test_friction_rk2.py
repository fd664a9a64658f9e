"""The two optional physics variants of the reference: the TYPE1 friction
patch of the resistance table (Stokes::setFriction, Stokes.cc:1132-1191) and
the two-stage Runge-Kutta integrator (Integrator.cu:232-438).

* The patched table from the library (fsd_resistance_table, host only) equals
  the oracle's restatement bit for bit, and differs from the plain table
  exactly in the patched entries of the rows within h0.
* R_FU with friction on the GPU against the oracle's R_FU on the patched
  table: 1e-5.
* One Runge-Kutta step at kT = 0 with shear, a squirmer term and directors
  against the oracle's two stages and the oracle's velocities at x and at the
  predictor: displacements 1e-4, directors 1e-5, images exactly, and the
  reported velocity (the mean of the stages) 1e-4 (GMRES to 1e-6).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import ewald_golden
from fsd_b200 import _lib
from fsd_b200.configs import suspension
from fsd_b200.core import FSD, default_params
from oracle import fsd_oracle as O

H0, ALPHA = 0.05, (0.5, 0.3, 0.2, 0.1, 0.4, 0.25)


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _table(friction):
    p = default_params()
    p.N, p.Lx, p.Ly, p.Lz = 10, 20.0, 20.0, 20.0
    if friction:
        p.friction_type, p.friction_h0 = 1, H0
        for k, a in enumerate(ALPHA):
            p.friction_alpha[k] = a
    d = np.zeros(1000, np.float32)
    v = np.zeros(22000, np.float32)
    assert _lib.lib().fsd_resistance_table(C.byref(p), d.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)) == 0
    return d, v.reshape(1000, 22)


def test_friction_table_equals_oracle_bit_for_bit():
    d0, v0 = _table(False)
    d1, v1 = _table(True)
    td, tv = O.resistance_table()
    assert np.array_equal(d0, td) and np.array_equal(v0, tv)
    ref = O.friction_table(td, tv, H0, ALPHA)
    assert np.array_equal(v1.view(np.uint32), ref.view(np.uint32))
    rows = (d1 - 2.0).astype(np.float32) <= np.float32(H0)
    changed = v1 != v0
    assert changed[rows][:, [3, 4, 5, 6, 9, 10]].all()
    assert not changed[~rows].any() and not changed[:, [0, 1, 2, 7, 8] + list(range(11, 22))].any()


@pytest.mark.gpu
def test_rfu_with_friction_matches_oracle(cuda):
    N = 400
    pos, Lc = suspension(N, 0.45, 12)
    L = (Lc, Lc, Lc)
    s = FSD(N, (Lc, Lc, Lc, 0.0), friction_type=1, friction_h0=H0, friction_alpha=(C.c_float * 6)(*ALPHA))
    p = torch.as_tensor(pos).cuda().view(-1).contiguous()
    s.build_neighbor_list(p)
    U = np.random.default_rng(3).standard_normal(6 * N)
    got = s.rfu(p, torch.as_tensor(U, dtype=torch.float32).cuda()).cpu().numpy()
    td, tv = O.resistance_table()
    rows = O.neighbor_list(pos, L, 0.0, s.pse_info().ewald_cut + 0.4)
    ref = O.rfu(pos, U, L, 0.0, rows, td, O.friction_table(td, tv, H0, ALPHA))
    plain = O.rfu(pos, U, L, 0.0, rows, td, tv)
    assert rel(got, ref) < 1e-5
    assert rel(plain, ref) > 1e-4  # the patch matters at this density
    s.close()


@pytest.mark.gpu
def test_runge_kutta_step_matches_oracle(cuda):
    N, phi, seed, xy, rate, dt, B1 = 200, 0.3, 14, 0.05, 0.6, 5e-3, 0.4
    pos, Lc = suspension(N, phi, seed)
    L = (Lc, Lc, Lc)
    rng = np.random.default_rng(seed)
    ori = rng.standard_normal((N, 3))
    ori = (ori / np.linalg.norm(ori, axis=1, keepdims=True)).astype(np.float32)
    mask = rng.random(N).astype(np.float32)
    s = FSD(N, (Lc, Lc, Lc, xy), T=0.0, dt=dt, sqm_B1=B1, solver_tol=1e-6, gmres_max_iter=4000, precond="learned",
            integrator=1)
    p = torch.as_tensor(pos).cuda().view(-1).contiguous()
    o = torch.as_tensor(ori).cuda().view(-1).contiguous()
    img = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
    gb = p.clone()
    F = torch.zeros(6 * N, device="cuda")
    V = torch.zeros(11 * N, device="cuda")
    s.step(0, rate, p, o, img, F, V, pos_gb=gb, b1_mask=torch.as_tensor(mask).cuda())
    table = ewald_golden()
    U1, _, _ = O.Problem(pos, L, xy, table=table).velocity(rate, tol=1e-11)
    ps, os_, gb1 = O.rk_stage1(pos, ori, pos, U1, dt, rate, B1=B1, b1mask=mask)
    psw, _ = O.wrap(ps, np.zeros((N, 3), np.int64), L, xy)
    U2, _, _ = O.Problem(psw, L, xy, table=table).velocity(rate, tol=1e-11)
    rp, rori, rgb, rimg = O.rk_stage2(pos, ori, ps, os_, gb1, U2, np.zeros((N, 3), np.int64), L, xy, dt, rate, B1=B1,
                                      b1mask=mask)
    got = p.cpu().numpy().reshape(N, 4)[:, :3].astype(np.float64)
    gimg = img.cpu().numpy().reshape(N, 3)
    assert np.array_equal(gimg, rimg)
    shift = lambda q, im: q + im * np.array(L) + np.stack([im[:, 1] * Lc * xy, 0 * im[:, 1], 0 * im[:, 1]], 1)
    assert rel(shift(got, gimg) - pos[:, :3], shift(rp, rimg) - pos[:, :3]) < 1e-4
    assert rel(o.cpu().numpy().reshape(N, 3), rori) < 1e-5
    assert rel(gb.cpu().numpy().reshape(N, 4)[:, :3], rgb[:, :3]) < 1e-5
    assert rel(V.cpu().numpy()[:6 * N], 0.5 * (U1 + U2)) < 1e-4
    s.close()
