"""Generate the golden fixtures in tests/golden from the reference itself.

Runs the reference's own code compiled for the host (oracle/_ref/libfsdref.so,
built by ``python oracle/ref_recipe/build_ref.py`` from the reference
checkout) on small seeded inputs and stores inputs and outputs as .npz/.json.
The fixtures let machines without the reference checkout (the GPU box) check
the oracle and the CUDA path against the reference's numbers.

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fsd_b200.configs import suspension  # noqa: E402
from oracle import fsd_oracle as O  # noqa: E402
from oracle import refbind as R  # noqa: E402

OUT = Path(__file__).resolve().parent


def wrap_sheared(pos, L, xy):
    """Wrap into the sheared box with fractional coordinates in [0, 1)."""
    p = np.asarray(pos, np.float64).copy()
    p[:, 2] -= L[2] * np.floor(p[:, 2] / L[2] + 0.5)
    ny = np.floor(p[:, 1] / L[1] + 0.5)
    p[:, 1] -= L[1] * ny
    p[:, 0] -= L[1] * xy * ny
    p[:, 0] -= L[0] * np.floor((p[:, 0] - xy * p[:, 1]) / L[0] + 0.5)
    out = np.zeros((len(p), 4), np.float32)
    out[:, :3] = p
    return out


def flat_rows(rows):
    return np.array([len(r) for r in rows], np.int64), np.concatenate([np.asarray(r, np.int64) for r in rows])


def pair_case(name, N, phi, xy, seed, shear_rate, B2, inject_close=False):
    pos, Lc = suspension(N, phi, seed)
    L = (Lc, Lc, Lc)
    rng = np.random.default_rng(seed + 100)
    if inject_close:
        # Pairs at the regularised contact (gap < 1e-3) and just inside r = 4.
        pos[1, :3] = pos[0, :3] + np.array([2.0005, 0.0, 0.0], np.float32)
        pos[3, :3] = pos[2, :3] + np.array([0.0, 2.00003, 0.0], np.float32)
        pos[5, :3] = pos[4, :3] + np.array([0.0, 0.0, 3.999], np.float32)
        pos[7, :3] = pos[6, :3] + np.array([2.9, 1.5, 0.4], np.float32)
    pos = wrap_sheared(pos[:, :3], L, xy)
    tab, sx, sy, cut, en = R.ewald_table(0.5, 1e-3)
    rows = O.neighbor_list(pos[:, :3], L, xy, cut + 0.4)
    tdist, tvals = O.resistance_table()
    genF = rng.standard_normal(11 * N).astype(np.float32)
    U6 = rng.standard_normal(6 * N).astype(np.float32)
    ori = rng.standard_normal((N, 3)).astype(np.float32)
    ori /= np.linalg.norm(ori, axis=1, keepdims=True)
    b2mask = (rng.random(N) < 0.5).astype(np.float32)
    # Real space through the reference kernel, in its float4 layouts.
    F4 = np.zeros((N, 4), np.float32)
    a = genF[: 6 * N].reshape(N, 6)
    s = genF[6 * N:].reshape(N, 5)
    F4[:, :3] = a[:, :3]
    TS = np.zeros((N, 8), np.float32)
    TS[:, :3] = a[:, 3:]
    TS[:, 3:] = s
    C8 = R.ts2c(TS)
    vel, delu = R.realspace(pos, F4, C8, rows, L, xy, 0.5, tab, sx, sy, cut, en)
    nn, flat = flat_rows(rows)
    np.savez_compressed(
        OUT / f"{name}.npz", pos=pos, L=np.array(L), xy=xy, genF=genF, U6=U6, ori=ori, b2mask=b2mask,
        shear_rate=shear_rate, B2=B2, nn=nn, flat=flat, couplet=C8, real_vel=vel, real_delu=delu,
        rfu=R.rfu(pos, U6, rows, L, xy, tdist, tvals),
        rfe=R.rfe(pos, shear_rate, rows, L, xy, tdist, tvals, ori, b2mask, B2),
        rsu=R.rsu(pos, U6, rows, L, xy, tdist, tvals),
        rse=R.rse(pos, shear_rate, rows, L, xy, tdist, tvals, ori, b2mask, B2),
        force=R.setforce(pos, ori, rows, L, xy, T_ext=0.7),
        strain_rhs=R.add_strain_rate(np.zeros(17 * N, np.float32), shear_rate, N, ori, b2mask, B2),
    )
    return pos, L, xy, rows, tdist, tvals


def precond_case(name, pos, L, xy, rows, tdist, tvals):
    r, c, v, prow = R.precond_coo(pos, rows, L, xy, tdist, tvals)
    perm = R.genrcm([np.asarray(p, np.int64) for p in prow])
    nn, flat = flat_rows(prow)
    np.savez_compressed(OUT / f"{name}.npz", coo_row=r, coo_col=c, coo_val=v, pn=nn, pflat=flat, rcm_perm=perm)


def grid_case(name, Nxyz, L, xy, seed):
    rng = np.random.default_rng(seed)
    gp = R.setparams(0.5, 1e-3, 0.5, L)
    gk = R.gridk(Nxyz, L, xy, 0.5, gp["eta"])
    G = int(np.prod(Nxyz))
    real = rng.standard_normal((11, G)).astype(np.float32)
    spec = np.fft.fftn(real.reshape(11, *Nxyz), axes=(1, 2, 3)).reshape(11, G).astype(np.complex64)
    out = R.green(spec, gk)
    noise = rng.standard_normal(6 * G + 8).astype(np.float32)
    np.savez_compressed(OUT / f"{name}.npz", Nxyz=np.array(Nxyz), L=np.array(L), xy=xy, eta=gp["eta"], gridk=gk,
                        spec_in=spec, spec_out=out, real_in=real)


def motion_case(name, seed):
    rng = np.random.default_rng(seed)
    N = 50
    L = (12.0, 12.0, 12.0)
    xy = 0.25
    pos = wrap_sheared(rng.uniform(-6, 6, (N, 3)), L, xy)
    ori = rng.standard_normal((N, 3)).astype(np.float32)
    ori /= np.linalg.norm(ori, axis=1, keepdims=True)
    vel = (rng.standard_normal(11 * N) * 50).astype(np.float32)
    gb = pos.copy()
    img = np.zeros((N, 3), np.int32)
    b1 = rng.random(N).astype(np.float32)
    noise = rng.standard_normal((N, 3)).astype(np.float32)
    p2, o2, g2, i2 = R.euler_shear(pos, ori, gb, vel, img, L, xy, 1e-2, 0.8, B1=0.3, b1mask=b1, noise=noise)
    np.savez_compressed(OUT / f"{name}.npz", pos=pos, ori=ori, vel=vel, gb=gb, b1mask=b1, noise=noise, L=np.array(L),
                        xy=xy, dt=1e-2, shear_rate=0.8, B1=0.3, pos_out=p2, ori_out=o2, gb_out=g2, img_out=i2)


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libfsdref.so missing: run python oracle/ref_recipe/build_ref.py")
    setups = []
    for N, phi, xi, err, ms in [(1000, 0.2, 0.5, 1e-3, 0.5), (32768, 0.4, 0.5, 1e-3, 0.5), (131072, 0.3, 0.5, 1e-3, 0.5),
                                (32768, 0.5, 0.5, 1e-3, 0.5), (4096, 0.3, 0.5, 1e-3, 0.5), (500, 0.3, 0.6, 1e-4, 0.2),
                                (2000, 0.1, 0.45, 5e-3, 0.0)]:
        L = (4 * np.pi * N / (3 * phi)) ** (1 / 3)
        for Lv in [(L, L, L), (L, 0.8 * L, 1.3 * L)]:
            ref = R.setparams(xi, err, ms, Lv)
            setups.append(dict(xi=xi, error=err, max_strain=ms, L=list(map(float, Lv)), ref=ref))
    (OUT / "setparams.json").write_text(json.dumps(setups, indent=1))
    tab, sx, sy, cut, en = R.ewald_table(0.5, 1e-3)
    np.savez_compressed(OUT / "ewald_xi0.5_err1e-3.npz", table=tab, self_x=sx, self_y=sy, cut=cut, n=en)
    tab2, sx2, sy2, cut2, en2 = R.ewald_table(0.8, 1e-4)
    np.savez_compressed(OUT / "ewald_xi0.8_err1e-4.npz", table=tab2, self_x=sx2, self_y=sy2, cut=cut2, n=en2)
    pair_case("pairs_dilute", 64, 0.15, 0.0, 11, 1.3, 0.0)
    pos, L, xy, rows, tdist, tvals = pair_case("pairs_dense_sheared", 200, 0.45, 0.3, 12, -0.7, 0.9, inject_close=True)
    precond_case("precond_dense_sheared", pos, L, xy, rows, tdist, tvals)
    grid_case("green_even", (12, 12, 12), (12.3, 12.3, 12.3), 0.0, 21)
    grid_case("green_mixed_sheared", (10, 9, 12), (12.3, 11.0, 13.1), 0.35, 22)
    motion_case("motion", 31)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
