"""FP64 NumPy restatement of the learned preconditioner -- TEST INFRASTRUCTURE ONLY.

Checker for fsd_b200/csrc/mpnn.cu: the pair graph (the two-hop sets of the
sparse approximate inverse), the invariant edge features, the message-passing
network, the axisymmetric block head whose output corrects the approximate
inverse G ~ (R_FU^pruned + D)^-1, and the loss
    L = sum_p ||A G z_p - z_p||^2 / (P 6N)
(training draws z = w - A G0 w from the residuals of the uncorrected G0).
The network has no counterpart in the reference; A is the reference's pruned
preconditioner matrix (Precondition.cu:530-836 plus the identity shift of
Helper_Precondition.cu:535-580), restated in fsd_oracle.pruned_rfu_sparse.
Gradients are checked against central differences of `loss` in FP64.
"""
from __future__ import annotations

import numpy as np

from . import fsd_oracle as O

WIDTH, LAYERS, FEAT, HEAD_E, HEAD_N = 64, 3, 16, 16, 16


def layout():
    """Offsets of the flat weight vector (fsd_mpnn.h MpLayout)."""
    o = {}
    k = 0
    def take(name, n):
        nonlocal k
        o[name] = (k, n)
        k += n
    take("W_in", WIDTH * FEAT)
    take("b_in", WIDTH)
    for l in range(LAYERS):
        take(f"W_m{l}", WIDTH * 3 * WIDTH)
        take(f"b_m{l}", WIDTH)
        take(f"W_h{l}", WIDTH * 2 * WIDTH)
        take(f"b_h{l}", WIDTH)
    take("W_o", HEAD_E * 3 * WIDTH)
    take("b_o", HEAD_E)
    take("W_n", HEAD_N * WIDTH)
    take("b_n", HEAD_N)
    return o, k


def unpack(w):
    o, n = layout()
    assert len(w) == n
    shapes = {"W_in": (WIDTH, FEAT), "W_o": (HEAD_E, 3 * WIDTH), "W_n": (HEAD_N, WIDTH)}
    for l in range(LAYERS):
        shapes[f"W_m{l}"] = (WIDTH, 3 * WIDTH)
        shapes[f"W_h{l}"] = (WIDTH, 2 * WIDTH)
    out = {}
    for name, (k, m) in o.items():
        v = np.asarray(w[k:k + m], np.float64)
        out[name] = v.reshape(shapes[name]) if name in shapes else v
    return out


def init_weights(seed=0, head_scale=1e-3):
    """He-initialised hidden layers, near-zero heads (G starts at the block-Jacobi inverse)."""
    rng = np.random.default_rng(seed)
    o, n = layout()
    w = np.zeros(n, np.float32)
    for name, (k, m) in o.items():
        if name.startswith("b"):
            continue
        fan_in = {"W_in": FEAT, "W_o": 3 * WIDTH, "W_n": WIDTH}.get(name, 3 * WIDTH if name.startswith("W_m") else 2 * WIDTH)
        scale = head_scale if name in ("W_o", "W_n") else np.sqrt(2.0 / fan_in)
        w[k:k + m] = rng.standard_normal(m) * scale
    return w


def graph(pos, L, xy, sets, prow):
    """Directed pairs c -> s for s != c in c's two-hop set, single-precision
    separations as the kernels; `direct` marks pairs in each other's pruned list."""
    p = np.asarray(pos, np.float32)[:, :3]
    i = np.array([c for c, S in enumerate(sets) for s in S[1:]], np.int64)
    j = np.array([s for c, S in enumerate(sets) for s in S[1:]], np.int64)
    R = O.min_image32(p[j] - p[i], L, xy)
    d2 = R[:, 0] * R[:, 0] + R[:, 1] * R[:, 1] + R[:, 2] * R[:, 2]
    d = np.sqrt(d2.astype(np.float32)).astype(np.float64)
    direct = np.array([s in prow[c] for c, s in zip(i, j)], bool)
    return i, j, R.astype(np.float64) / d[:, None], d, direct


def features(d, direct, tdist, tvals):
    h = d - 2.0
    c = O.res_interp(d, 0, 10, tdist, tvals, mode="lub")
    x = np.zeros((len(d), FEAT))
    x[:, 0] = np.log(np.maximum(h, 1e-4)) * 0.2
    x[:, 1] = h
    x[:, 2] = np.exp(-10.0 * np.maximum(h, 0.0))
    x[:, 3] = 2.0 / d
    x[:, 4:14] = np.sign(c) * np.log1p(np.abs(c)) * 0.25
    x[:, 14] = direct
    x[:, 15] = 1.0
    return x


def segmean(v, i, N):
    out = np.zeros((N, v.shape[1]))
    np.add.at(out, i, v)
    deg = np.bincount(i, minlength=N).astype(np.float64)
    return out / np.maximum(deg, 1)[:, None]


def forward(wv, x, i, j, N):
    P = unpack(wv)
    relu = lambda z: np.maximum(z, 0.0)
    e = relu(x @ P["W_in"].T + P["b_in"])
    h = segmean(e, i, N)
    for l in range(LAYERS):
        m = relu(np.concatenate([e, h[i], h[j]], 1) @ P[f"W_m{l}"].T + P[f"b_m{l}"])
        e = e + m
        a = segmean(m, i, N)
        h = h + relu(np.concatenate([h, a], 1) @ P[f"W_h{l}"].T + P[f"b_h{l}"])
    oe = np.concatenate([e, h[i], h[j]], 1) @ P["W_o"].T + P["b_o"]
    on = h @ P["W_n"].T + P["b_n"]
    return oe, on


def axis_block(o, r):
    """B(o, r) = [o0 rr + o1 (I - rr), o2 [r]x ; o3 [r]x, o4 rr + o5 (I - rr)] per row."""
    n = len(r)
    rr = r[:, :, None] * r[:, None, :]
    I = np.eye(3)[None]
    cx = np.zeros((n, 3, 3))
    cx[:, 0, 1], cx[:, 0, 2] = -r[:, 2], r[:, 1]
    cx[:, 1, 0], cx[:, 1, 2] = r[:, 2], -r[:, 0]
    cx[:, 2, 0], cx[:, 2, 1] = -r[:, 1], r[:, 0]
    w = lambda k: o[:, k][:, None, None]
    B = np.zeros((n, 6, 6))
    B[:, :3, :3] = w(0) * rr + w(1) * (I - rr)
    B[:, :3, 3:] = w(2) * cx
    B[:, 3:, :3] = w(3) * cx
    B[:, 3:, 3:] = w(4) * rr + w(5) * (I - rr)
    return B


def g_blocks(oe, on, J, i, rhat, N):
    """Correction blocks dG_ij = J_i B(o_ij) and dG_ii = J_i (iso + sum_j B(q_ij))."""
    Ge = np.einsum("nab,nbc->nac", J[i], axis_block(oe[:, :6], rhat))
    S = np.zeros((N, 6, 6))
    np.add.at(S, i, axis_block(oe[:, 6:12], rhat))
    d = np.concatenate([np.repeat(on[:, :1], 3, 1), np.repeat(on[:, 1:2], 3, 1)], 1)
    S[:, np.arange(6), np.arange(6)] += d
    Gs = np.einsum("nab,nbc->nac", J, S)
    return Ge, Gs


def problem(pos, L, xy):
    """Everything the loss needs that does not depend on the weights."""
    import scipy.sparse as sp
    tdist, tvals = O.resistance_table()
    N = len(pos)
    A = O.pruned_rfu_sparse(pos, L, xy, tdist, tvals, rows=O.neighbor_list(pos, L, xy, 6.0)).tocsr()
    Ab = sp.bsr_matrix(A, blocksize=(6, 6))
    Ab.sort_indices()
    sets = O.spai_sets(Ab, N)
    prow = [set(int(k) for k in Ab.indices[Ab.indptr[c]:Ab.indptr[c + 1]]) for c in range(N)]
    J = np.stack([np.linalg.inv(A[6 * k:6 * k + 6, 6 * k:6 * k + 6].toarray()) for k in range(N)])
    i, j, rhat, d, direct = graph(pos, L, xy, sets, prow)
    x = features(d, direct, tdist, tvals)
    return dict(N=N, A=A, G0=O.spai2(A, N), J=J, i=i, j=j, rhat=rhat, x=x)


def g_matrix(wv, pr):
    import scipy.sparse as sp
    N, i, j = pr["N"], pr["i"], pr["j"]
    oe, on = forward(wv, pr["x"], i, j, N)
    Ge, Gs = g_blocks(oe, on, pr["J"], i, pr["rhat"], N)
    rows = np.concatenate([i, np.arange(N)])
    cols = np.concatenate([j, np.arange(N)])
    blocks = np.concatenate([Ge, Gs])
    ri = (6 * rows[:, None, None] + np.arange(6)[None, :, None]) * np.ones((1, 1, 6), np.int64)
    ci = (6 * cols[:, None, None] + np.arange(6)[None, None, :]) * np.ones((1, 6, 1), np.int64)
    dG = sp.csr_matrix((blocks.ravel(), (ri.ravel(), ci.ravel())), shape=(6 * N, 6 * N))
    return pr["G0"] + dG


def loss(wv, pr, Z):
    """Z: probes (P, 6N)."""
    G = g_matrix(wv, pr)
    R = (pr["A"] @ (G @ Z.T)).T - Z
    return float(np.sum(R * R) / (Z.shape[0] * 6 * pr["N"]))


# ------------------------------------------------ learned inner polynomial
def cheb_images(A, G, T, lam, k):
    """W_m = A G T_m(S) t for m < k, S = (2/lam) A G - I, probes T (P, 6N);
    returns (k, 6N, P)."""
    B = [T.T]
    W = []
    for m in range(k):
        Wm = A @ (G @ B[m])
        W.append(Wm)
        if m + 1 < k:
            if m == 0:
                B.append((2.0 / lam) * Wm - B[0])
            else:
                B.append(2.0 * ((2.0 / lam) * Wm - B[m]) - B[m - 1])
    return np.stack(W)


def poly_coeffs(wv, pr, k):
    """Chebyshev coefficients the network predicts: mean over particles of the
    node head's first k outputs (mpnn.cu k_poly_pool)."""
    _, on = forward(wv, pr["x"], pr["i"], pr["j"], pr["N"])
    return on[:, :k].mean(0)


def poly_loss_c(c, W, T):
    """E_t ||t - sum_m c_m W_m t||^2 / ||t||^2 over the probes."""
    R = T.T - np.einsum("m,mnp->np", c, W)
    return float(np.mean(np.sum(R * R, 0) / np.sum(T.T * T.T, 0)))


def poly_loss(wv, pr, T, lam, k):
    return poly_loss_c(poly_coeffs(wv, pr, k), cheb_images(pr["A"], pr["G0"], T, lam, k), T)


def poly_apply(b, c, lam, A, G, N):
    """Saddle preconditioner with y = G q(AG) t, q = sum c_m T_m(2x/lam - 1),
    evaluated in FP64 by Clenshaw's recurrence (poly.cu)."""
    b = np.asarray(b, np.float64)
    t = b[: 6 * N] - b[11 * N:]
    k = len(c)
    S = lambda v: (2.0 / lam) * (A @ (G @ v)) - v
    b1 = c[k - 1] * t
    b2 = np.zeros_like(t)
    for m in range(k - 2, 0, -1):
        b1, b2 = c[m] * t + 2.0 * S(b1) - b2, b1
    v = c[0] * t + S(b1) - b2
    y = G @ v
    x = b.copy()
    x[: 6 * N] = b[: 6 * N] - y
    x[11 * N:] = y
    return x


def interval_coefficients(rho, k):
    """Coefficients c_m (m < k, lambda = 1) of q in T_m(2u - 1) with
    1 - u q(u) = T_k((1 + rho - 2u)/(1 - rho)) / T_k((1 + rho)/(1 - rho)):
    FP64 least squares on 64 points, an independent route to the library's
    interpolation."""
    def T(n, z):
        z = np.asarray(z, np.float64)
        out = np.empty_like(z)
        m = np.abs(z) <= 1
        out[m] = np.cos(n * np.arccos(z[m]))
        zz = z[~m]
        out[~m] = np.cosh(n * np.arccosh(np.abs(zz))) * np.where((zz < 0) & (n % 2 == 1), -1.0, 1.0)
        return out
    u = np.linspace(0.01, 1.0, 64)
    r = T(k, (1 + rho - 2 * u) / (1 - rho)) / T(k, np.array([(1 + rho) / (1 - rho)]))[0]
    q = (1 - r) / u
    B = np.stack([T(m, 2 * u - 1) for m in range(k)], 1)
    c, *_ = np.linalg.lstsq(B, q, rcond=None)
    return c


def ratio_loss(wv, pr, target):
    """(log rho prediction - target)^2 with log rho = mean of the node head's first output."""
    _, on = forward(wv, pr["x"], pr["i"], pr["j"], pr["N"])
    return float((on[:, 0].mean() - target) ** 2)
