"""Seeded synthetic suspensions of unit spheres in a cubic periodic box.

Random sequential addition (RSA) with a minimum surface gap places particles
until insertion stalls (RSA jams near phi ~ 0.38); any remaining particles are
then inserted at random and overlaps are relaxed by pairwise separation
sweeps, the "RSA then overlap-relaxation" recipe the benchmark configurations
call for.  Positions are float32, box centred on the origin.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.spatial import cKDTree


def box_length(N: int, phi: float) -> float:
    """L = (4 pi N / (3 phi))^(1/3) for unit spheres."""
    return (4.0 * math.pi * N / (3.0 * phi)) ** (1.0 / 3.0)


def _wrap(x, L):
    return x - L * np.floor(x / L)


def rsa(N: int, L: float, rng: np.random.Generator, min_gap: float = 1e-3, max_rounds: int = 200) -> np.ndarray:
    """Batch RSA in [0, L)^3; returns as many particles as could be placed (<= N)."""
    dmin = 2.0 + min_gap
    pos = np.zeros((0, 3))
    for _ in range(max_rounds):
        need = N - len(pos)
        if need <= 0:
            break
        cand = rng.random((min(4 * need + 64, 200000), 3)) * L
        if len(pos):
            tree = cKDTree(pos, boxsize=L)
            d, _ = tree.query(cand, k=1)
            cand = cand[d >= dmin]
        if len(cand) == 0:
            continue
        ct = cKDTree(cand, boxsize=L)
        pairs = ct.query_pairs(dmin, output_type="ndarray")
        ok = np.ones(len(cand), bool)
        if len(pairs):
            # Greedy in candidate order: drop the later member of each conflicting pair.
            order = np.argsort(pairs[:, 0], kind="stable")
            for a, b in pairs[order]:
                if ok[a] and ok[b]:
                    ok[b] = False
        acc = cand[ok][:need]
        if len(acc) == 0:
            break
        pos = np.concatenate([pos, acc])
        if len(acc) < 0.01 * need and len(pos) < N:
            break
    return pos


def relax_overlaps(pos: np.ndarray, L: float, min_gap: float = 1e-3, sweeps: int = 200, target_gap: float | None = None,
                   factor: float = 1.02) -> np.ndarray:
    """Separate pairs closer than the minimum gap along their line of centres
    (each by `factor` times half the shortfall to `target_gap`, default the
    minimum gap) until the minimum gap holds or the sweep budget runs out."""
    dmin = 2.0 + min_gap
    dpush = 2.0 + (min_gap if target_gap is None else target_gap)
    pos = pos.copy()
    for _ in range(sweeps):
        tree = cKDTree(_wrap(pos, L), boxsize=L)
        if len(tree.query_pairs(dmin, output_type="ndarray")) == 0:
            break
        pairs = tree.query_pairs(dpush, output_type="ndarray")
        d = pos[pairs[:, 1]] - pos[pairs[:, 0]]
        d -= L * np.rint(d / L)
        r = np.linalg.norm(d, axis=1)
        r = np.maximum(r, 1e-9)
        push = 0.5 * (dpush - r)[:, None] * d / r[:, None] * factor
        disp = np.zeros_like(pos)
        np.add.at(disp, pairs[:, 0], -push)
        np.add.at(disp, pairs[:, 1], push)
        pos = _wrap(pos + disp, L)
    return pos


def suspension(N: int, phi: float, seed: int, min_gap: float = 1e-3, relax_sweeps: int = 200):
    """Positions (N,4) float32 (w = 0) centred on the origin, and the box edge L."""
    L = box_length(N, phi)
    rng = np.random.default_rng(seed)
    pos = rsa(N, L, rng, min_gap)
    if len(pos) < N:
        pos = np.concatenate([pos, rng.random((N - len(pos), 3)) * L])
    pos = relax_overlaps(pos, L, min_gap, relax_sweeps)
    if min_gap_f64(pos, L) < 0.0:
        # overlaps left (phi above about 0.5): push pairs toward three times
        # the gap, one and a half times the shortfall per sweep, until it holds
        pos = relax_overlaps(pos, L, min_gap, 1000, target_gap=3 * min_gap, factor=1.5)
    pos = _wrap(pos, L) - L / 2.0
    out = np.zeros((N, 4), np.float32)
    out[:, :3] = pos
    # Keep float32 coordinates strictly inside [-L/2, L/2).
    x = out[:, :3]
    x[x >= np.float32(L / 2.0)] -= np.float32(L)
    return out, L


def min_gap_f64(pos: np.ndarray, L: float) -> float:
    """Smallest surface gap of positions in [0, L)^3 (or any periodic image)."""
    p = _wrap(np.asarray(pos, np.float64)[:, :3], L)
    d, _ = cKDTree(p, boxsize=L).query(p, k=2)
    return float(d[:, 1].min() - 2.0)


def min_gap(pos: np.ndarray, L: float) -> float:
    p = _wrap(np.asarray(pos, np.float64)[:, :3], L)
    d, _ = cKDTree(p, boxsize=L).query(p, k=2)
    return float(d[:, 1].min() - 2.0)
