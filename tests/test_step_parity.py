"""The parts of a time step that follow the solve, and one whole Brownian step,
against the FP64 oracle.

* Euler + shear (Integrator_ExplicitEuler_Shear_kernel, Integrator.cu:126-228)
  through fsd_integrate_euler: a sheared, tilted box with particles pushed
  across every face, nonzero starting images, unwrapped positions, a squirmer
  B1 term with a per-particle mask and angular noise.  Positions to 2e-6 of
  the box edge (FP32 coordinates), images exactly, directors and unwrapped
  positions to 1e-5 relative.
* The random finite difference drift (Integrator.cu:549-718) for the same
  drift direction psi (fsd_draw_normals, stream 4): (kT/eps)(U(x + eps psi/2)
  - U(x - eps psi/2)) with A(x') U = (0; -psi), solved by the oracle at the
  same FP32 displaced positions.  The difference of two solutions divided by
  eps = 1e-3 amplifies the solver residual (1e-6 here, just above the FP32
  residual floor of these right-hand sides) and FP32 rounding of the operator
  by 1e3, so the bar is 5e-3.
* One full step at kT = 1 with shear (fsd_step, Stokes_StepOne, Stokes.cu:119)
  against the oracle's right-hand side, saddle solve, stresslet and Euler
  update, given the library's own Brownian vectors for that step (far-field
  slip, near-field force and drift: fsd_brownian_farfield / _nearfield /
  fsd_rfd_drift at the same timestep on a fresh handle, which draw the same
  counter-based normals).  Once without and once with the active terms
  (squirmer B1/B2 with masks, rotational noise, external torque).  Velocities
  and stresslets to 1e-4 (GMRES to 3e-6; the random finite difference solves
  of this sheared, tilted case may stop at their FP32 residual floor a little
  above it, which the library reports, and the check uses the library's own
  drift), displacements to 1e-4, images exactly.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import ewald_golden
from fsd_b200 import _lib
from fsd_b200.configs import suspension
from fsd_b200.core import FSD
from oracle import fsd_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def dev(x, dtype=np.float32):
    return torch.as_tensor(np.ascontiguousarray(x, dtype)).cuda().contiguous().view(-1)


def test_euler_shear_matches_oracle(cuda):
    rng = np.random.default_rng(31)
    N, Lc, xy, dt, rate, B1 = 1000, 20.0, 0.3, 1e-2, 0.8, 0.7
    L = (Lc, Lc, Lc)
    pos = np.zeros((N, 4), np.float32)
    pos[:, 1:3] = (rng.random((N, 2)) - 0.5) * Lc * 0.999
    pos[:, 0] = (rng.random(N) - 0.5) * Lc * 0.999 + xy * pos[:, 1]
    vel = np.zeros(11 * N, np.float32)
    v6 = vel[:6 * N].reshape(N, 6)
    v6[:, :3] = rng.standard_normal((N, 3)) * (0.4 * Lc / dt)   # large enough to cross faces
    v6[:, 3:] = rng.standard_normal((N, 3)) * 20.0
    ori = rng.standard_normal((N, 3))
    ori = (ori / np.linalg.norm(ori, axis=1, keepdims=True)).astype(np.float32)
    img = rng.integers(-3, 4, (N, 3)).astype(np.int32)
    gb = np.zeros((N, 4), np.float32)
    gb[:, :3] = pos[:, :3] + img * Lc
    mask = rng.random(N).astype(np.float32)
    noise = (rng.standard_normal((N, 3)) * 5.0).astype(np.float32)
    s = FSD(N, (Lc, Lc, Lc, xy), dt=dt, sqm_B1=B1)
    p, o, g, im = dev(pos), dev(ori), dev(gb), dev(img, np.int32)
    s.integrate_euler(0, rate, p, o, im, dev(vel), pos_gb=g, noise_ang=dev(noise), b1_mask=dev(mask))
    rp, rori, rgb, rimg = O.euler_shear(pos, ori, gb, vel, img, L, xy, dt, rate, B1=B1, b1mask=mask, noise=noise)
    got_p = p.cpu().numpy().reshape(N, 4)[:, :3]
    assert np.abs(got_p - rp).max() < 2e-6 * Lc
    assert np.array_equal(im.cpu().numpy().reshape(N, 3), rimg)
    assert rel(o.cpu().numpy().reshape(N, 3), rori) < 1e-5
    assert rel(g.cpu().numpy().reshape(N, 4)[:, :3], rgb[:, :3]) < 1e-5
    moved = np.abs(rimg - img).sum()
    assert moved > N // 4  # the case exercises the wraps
    s.close()


def _displaced32(pos, psi, d, L, xy):
    """k_displace in FP32: x + d psi, then one wrap per axis."""
    N = len(pos)
    x = (pos[:, :3].astype(np.float32) + psi.reshape(N, 6)[:, :3].astype(np.float32) * np.float32(d))
    x, _ = O.wrap(x, np.zeros((N, 3), np.int64), tuple(np.float32(v) for v in L), np.float32(xy))
    out = np.zeros((N, 4), np.float32)
    out[:, :3] = x
    return out


def test_rfd_drift_matches_oracle(cuda):
    N, phi, seed, eps, T = 200, 0.3, 5, 1e-3, 1.0
    pos, Lc = suspension(N, phi, seed)
    L = (Lc, Lc, Lc)
    s = FSD(N, (Lc, Lc, Lc, 0.0), T=T, dt=1e-4, seed=9, rfd_epsilon=eps, solver_tol=1e-6, gmres_max_iter=4000,
            precond="learned")
    p = dev(pos)
    img = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
    s.build_neighbor_list(p)
    s.precond_build(p)
    drift = s.rfd_drift(p, img, 4).cpu().numpy()
    psi = s.draw_normals(4, 4, 6 * N).cpu().numpy().astype(np.float64)
    U = []
    for sign in (+1, -1):
        xp = _displaced32(pos, psi, sign * eps / 2, L, 0.0)
        pr = O.Problem(xp, L, 0.0, table=ewald_golden())
        rhs = np.zeros(17 * N)
        rhs[11 * N:] = -psi
        U.append(pr.solve(rhs, tol=1e-11)[11 * N:])
    ref = (T / eps) * (U[0] - U[1])
    err = rel(drift, ref)
    print(f"RFD drift N={N}: rel err {err:.2e}")
    assert err < 5e-3
    s.close()


@pytest.mark.parametrize("active", [False, True])
def test_full_brownian_step_matches_oracle(cuda, active):
    N, phi, seed, xy, rate, dt, T = 200, 0.3, 8, 0.1, 0.7, 1e-3, 1.0
    pos, Lc = suspension(N, phi, seed)
    L = (Lc, Lc, Lc)
    rng = np.random.default_rng(seed)
    kw = dict(T=T, dt=dt, seed=11, solver_tol=3e-6, gmres_max_iter=4000, period=1, precond="learned",
              lanczos_tol=1e-4)
    ori = np.tile([0.0, 0.0, 1.0], (N, 1)).astype(np.float32)
    b1m = b2m = None
    if active:
        kw.update(sqm_B1=0.6, sqm_B2=0.4, rot_diff=0.3, T_ext=0.5, omega_ext=0.0)
        ori = rng.standard_normal((N, 3))
        ori = (ori / np.linalg.norm(ori, axis=1, keepdims=True)).astype(np.float32)
        b1m = rng.random(N).astype(np.float32)
        b2m = rng.random(N).astype(np.float32)
    # library's Brownian vectors for timestep 0 on a fresh handle
    sb = FSD(N, (Lc, Lc, Lc, xy), **kw)
    p0 = dev(pos)
    img0 = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
    sb.build_neighbor_list(p0)
    sb.precond_build(p0)
    UB = sb.brownian_farfield(p0, 0).cpu().numpy().astype(np.float64)
    FB = sb.brownian_nearfield(p0, 0).cpu().numpy().astype(np.float64)
    # the drift's two solves may stop at their FP32 residual floor (reported as
    # FSD_ERR_GMRES_MAXIT); the check below uses the library's own drift vector
    d_drift = torch.zeros(6 * N, device="cuda")
    st = _lib.lib().fsd_rfd_drift(sb._h, p0.data_ptr(), img0.data_ptr(), 0, d_drift.data_ptr())
    assert st in (0, 3) and max(sb.solve_info()["gmres_resid"][:2]) < 1e-5
    drift = d_drift.cpu().numpy().astype(np.float64)
    rot = sb.draw_normals(5, 0, 3 * N, float(np.sqrt(2 * kw.get("rot_diff", 0.0) / dt))).cpu().numpy()
    sb.close()
    # the full step on another fresh handle
    s = FSD(N, (Lc, Lc, Lc, xy), **kw)
    p = dev(pos)
    o = dev(ori)
    img = torch.zeros(3 * N, dtype=torch.int32, device="cuda")
    gb = dev(pos)
    F = torch.zeros(6 * N, device="cuda")
    V = torch.zeros(11 * N, device="cuda")
    st = s.step(0, rate, p, o, img, F, V, pos_gb=gb, b1_mask=None if b1m is None else dev(b1m),
                b2_mask=None if b2m is None else dev(b2m), raise_on_error=False)
    info = s.solve_info()
    assert st in (0, 3) and max(info["gmres_resid"]) < 1e-5
    v = V.cpu().numpy().astype(np.float64)
    # oracle: right-hand side, solve, stresslet, Euler
    pr = O.Problem(pos, L, xy, table=ewald_golden())
    B1, B2 = kw.get("sqm_B1", 0.0), kw.get("sqm_B2", 0.0)
    Fp = O.pair_force(pos, L, xy, pr.rows, T_ext=kw.get("T_ext", 0.0))
    assert rel(F.cpu().numpy(), Fp) < 1e-5
    rhs = O.strain_rhs(rate, N, ori=ori, b2mask=b2m, B2=B2)
    rhs[:11 * N] += UB
    rhs[11 * N:] += FB - Fp + O.rfe(pr.pos, rate, L, xy, pr.rows, pr.tdist, pr.tvals, ori=ori, b2mask=b2m, B2=B2)
    x = pr.solve(rhs, tol=1e-11)
    U = x[11 * N:] + drift
    S = x[6 * N:11 * N] + O.rsu(pr.pos, U, L, xy, pr.rows, pr.tdist, pr.tvals) \
        + O.rse(pr.pos, rate, L, xy, pr.rows, pr.tdist, pr.tvals, ori=ori, b2mask=b2m, B2=B2)
    eu, es = rel(v[:6 * N], U), rel(v[6 * N:], S)
    print(f"full step active={active}: velocity rel err {eu:.2e}, stresslet rel err {es:.2e}, "
          f"GMRES {s.solve_info()['gmres_iters']} residuals {s.solve_info()['gmres_resid']}")
    assert eu < 1e-4 and es < 1e-4
    noise = rot.reshape(N, 3) if active else None
    rp, rori, rgb, rimg = O.euler_shear(pos, ori, pos, U, np.zeros((N, 3), np.int64), L, xy, dt, rate, B1=B1,
                                        b1mask=b1m, noise=noise)
    got = p.cpu().numpy().reshape(N, 4)[:, :3].astype(np.float64)
    gimg = img.cpu().numpy().reshape(N, 3)
    assert np.array_equal(gimg, rimg)
    # displacement, unwrapped through the images
    d_got = got + gimg * np.array(L) - pos[:, :3]
    d_ref = rp + rimg * np.array(L) - pos[:, :3]
    d_got[:, 0] += gimg[:, 1] * Lc * xy
    d_ref[:, 0] += rimg[:, 1] * Lc * xy
    assert rel(d_got, d_ref) < 1e-4
    assert rel(o.cpu().numpy().reshape(N, 3), rori) < 1e-5
    assert rel(gb.cpu().numpy().reshape(N, 4)[:, :3], rgb[:, :3]) < 1e-5
    s.close()
