"""Per-particle text output of the reference's Stokes::OutputData
(Stokes.cc:703-931), host side: files raw/stresslet.<step>.txt,
raw/position.<step>.txt, raw/velocity.<step>.txt,
raw/interparticle_stresslet.<step>.txt and the appended overlap.txt, with
the same columns and printf formats.  Particles are written in index order
(tags equal indices here).  Where the reference aborts on an overlap larger
than 0.1, this raises RuntimeError."""
from __future__ import annotations

from pathlib import Path

import numpy as np


def _min_image(d, box):
    Lx, Ly, Lz, xy = box
    d = d.copy()
    img = np.rint(d[..., 2] / Lz)
    d[..., 2] -= Lz * img
    img = np.rint(d[..., 1] / Ly)
    d[..., 0] -= Ly * xy * img
    d[..., 1] -= Ly * img
    d[..., 0] -= Lx * np.rint(d[..., 0] / Lx)
    return d


def pair_stats(pos, box, rlist, pair):
    """Overlap statistics and interparticle stresslets over pairs closer than rlist."""
    p = np.asarray(pos, np.float64)[:, :3]
    N = len(p)
    Lx, Ly, Lz, xy = box
    nden = N / (Lx * Ly * Lz)
    F0 = 1.0 / pair["ndsr"]
    H = F0 * pair["beta_AF"]
    epsq, kappa, k_n = pair["epsq"], pair["kappa"], pair["k_n"]
    S = np.zeros((N, 6))
    max_ov, sum_ov, cnt, min_gap = 0.0, 0.0, 0.0, 10.0
    for i in range(N):
        R = _min_image(p - p[i], box)
        d = np.sqrt(np.einsum("ij,ij->i", R, R))
        m = (d < rlist)
        m[i] = False
        for j in np.nonzero(m)[0]:
            gap = d[j] - 2.0
            if gap < 0.0:
                ov = -gap
                if ov > 0.1:
                    raise RuntimeError(f"large overlap {ov:.3e} between particles {i} and {j}")
                max_ov = max(max_ov, ov)
                sum_ov += ov
                cnt += 1.0
                min_gap = 0.0
            elif gap < min_gap:
                min_gap = gap
            if d[j] <= 2.0 + 10.0 / kappa:
                n = R[j] / d[j]
                gap1 = d[j] - (2.0 + np.sqrt(epsq))
                if gap1 >= 0.0:
                    f = -F0 * np.exp(-gap1 * kappa) + H / (12.0 * (gap1 * gap1 + epsq))
                else:
                    f = H / (12.0 * epsq) - F0 - k_n * abs(gap1)
                c = nden * f / 2.0
                S[i] += c * np.array([n[0] * R[j, 0], n[0] * R[j, 1], n[0] * R[j, 2],
                                      n[1] * R[j, 1], n[1] * R[j, 2], n[2] * R[j, 2]])
    avg = sum_ov / cnt if cnt > 0 else 0.0
    return S, (cnt / 2.0 if cnt > 0 else 0.0, max_ov, avg, min_gap), nden


def write_output(outdir, timestep, box, pos, ori, pos_gb, velocity, pair, rlist):
    outdir = Path(outdir)
    raw = outdir / "raw"
    raw.mkdir(parents=True, exist_ok=True)
    N = len(pos)
    S_int, (cnt, max_ov, avg_ov, min_gap), nden = pair_stats(pos, box, rlist, pair)
    vel = np.asarray(velocity, np.float32)
    st = vel[6 * N:11 * N].reshape(N, 5) * np.float32(nden)
    ts = f"{timestep:010d}"
    with open(raw / f"stresslet.{ts}.txt", "w") as f0, open(raw / f"position.{ts}.txt", "w") as f1, \
            open(raw / f"interparticle_stresslet.{ts}.txt", "w") as f3, open(raw / f"velocity.{ts}.txt", "w") as f4:
        for i in range(N):
            sxx, sxy, sxz, syz, syy = (float(v) for v in st[i])
            szz = -sxx - syy
            f0.write("%7i %12.3e %12.3e %12.3e %12.3e %12.3e %12.3e \n" % (i, sxx, sxy, sxz, syy, syz, szz))
            f1.write("%7i %15.6e %15.6e %15.6e %12.3e %12.3e %12.3e %15.6e %15.6e %15.6e \n" % (
                i, pos[i, 0], pos[i, 1], pos[i, 2], ori[i, 0], ori[i, 1], ori[i, 2],
                pos_gb[i, 0], pos_gb[i, 1], pos_gb[i, 2]))
            u = vel[6 * i:6 * i + 6]
            f4.write("%7i %15.6e %15.6e %15.6e %12.3e %12.3e %12.3e \n" % (i, *[float(v) for v in u]))
            f3.write("%7i %12.3e %12.3e %12.3e %12.3e %12.3e %12.3e \n" % (i, *S_int[i]))
    with open(outdir / "overlap.txt", "a") as f2:
        f2.write("%9i %8.0f %12.3e %12.3e  %12.3e \n" % (timestep, cnt, max_ov, avg_ov, min_gap))
