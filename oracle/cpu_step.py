"""Host-core timing of one FSD step with the FP64 oracle -- BASELINE INFRASTRUCTURE.

Used only by bench.py (its ``cpu_baseline`` leg and the ``--impl reference``
arm) to report what the same method costs on the host cores; it is never part
of the CUDA product path.

A full step at N = 32768 takes hours in FP64 NumPy, so every stage of the step
(Stokes_StepOne, Stokes.cu:119-273; Integrator_ComputeVelocity,
Integrator.cu:744-938) is timed once on the real configuration and the step is
assembled from those stage times and the operator counts of the IChol method:

  neighbour list      cell search over the configuration (cKDTree), r < r_cut + 0.4
  pair force          Helper_Stokes.cu:65-172
  preconditioner      pruned R_FU + D assembly (Precondition.cu:530-836) and its
                      incomplete factorisation (SciPy spilu with its default
                      drop tolerance, standing in for csric02 on the RCM order)
  wave-space noise    one wave-space pass of the mobility (spread, 11 FFTs,
                      Green, contract) as the cost of the random field's transform
  Lanczos (far)       real-space mobility applications (Brownian_FarField.cu:597-808)
  Lanczos (near)      R_FU applications (Brownian_NearField.cu:174-464)
  GMRES               saddle operator (Saddle.cu:80-151) + preconditioner
                      application (Saddle.cu:171-264) + Gram-Schmidt against
                      the Krylov basis at its mean depth, per iteration, for the
                      two RFD solves and the main solve (Integrator.cu:549-718, 876)
  Euler               Integrator.cu:126-228

FFTs run on all host cores (scipy.fft workers) and dense BLAS uses its
default threads; the pair sums are single-threaded NumPy.

`full_step_seconds` runs one complete step end to end instead (Lanczos to
convergence, the three GMRES solves to 1e-4), at sizes the FP64 oracle
finishes in seconds (N = 1000); bench.py reports it beside the assembled
full-size figure.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import fsd_oracle as O


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _timed(fn, *a, **k):
    t = time.perf_counter()
    out = fn(*a, **k)
    return out, time.perf_counter() - t


class StepSampler:
    """Stage times of one FP64 FSD step on one configuration."""

    def __init__(self, pos, L, table, threads: int | None = None, restart: int = 200):
        self.threads = threads or os.cpu_count() or 1
        O.FFT_WORKERS = self.threads
        self.pos = O.xyz(pos)
        self.N = len(self.pos)
        self.L = (float(L), float(L), float(L)) if np.isscalar(L) else tuple(float(v) for v in L)
        self.table = table
        self.restart = restart
        self.t = {}
        self.pr = None

    def _neighbor_rows(self):
        from scipy.spatial import cKDTree
        Lb = np.array(self.L)
        x = np.mod(self.pos + Lb / 2, Lb)
        rlist = self.table[3] + 0.4
        pairs = cKDTree(x, boxsize=Lb).query_pairs(rlist, output_type="ndarray")
        i = np.concatenate([pairs[:, 0], pairs[:, 1]])
        j = np.concatenate([pairs[:, 1], pairs[:, 0]])
        order = np.lexsort((j, i))
        i, j = i[order], j[order]
        starts = np.searchsorted(i, np.arange(self.N + 1))
        return [j[starts[k]:starts[k + 1]].astype(np.uint32) for k in range(self.N)]

    def sample_setup(self):
        """Per-step stages that run once: list, force, preconditioner build, noise, Euler."""
        import scipy.sparse.linalg as sla
        N = self.N
        rows, self.t["nlist"] = _timed(self._neighbor_rows)
        pr = O.Problem.__new__(O.Problem)  # the oracle's problem with the list above
        pr.pos, pr.N, pr.L, pr.xy, pr.xi = self.pos, N, self.L, 0.0, 0.5
        pr.gp = O.grid_params(0.5, 1e-3, 0.5, self.L)
        pr.table, pr.self_x, pr.self_y, pr.ewald_cut, pr.ewald_n = self.table
        pr.rows = rows
        pr.tdist, pr.tvals = O.resistance_table()
        pr.rlub, pr.rp, pr.pi_typo = 4.0, 2.1, True
        self.pr = pr
        _, self.t["pair_force"] = _timed(O.pair_force, self.pos, self.L, 0.0, rows)

        def build():
            A = O.pruned_rfu_sparse(self.pos, self.L, 0.0, pr.tdist, pr.tvals, rows=rows, rp=2.1).tocsc()
            return sla.spilu(A, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0)
        self.ilu, self.t["precond_build"] = _timed(build)
        rng = np.random.default_rng(0)
        pr.mobility(rng.standard_normal(11 * N), 1)  # untimed: FFT plans and first-touch allocations
        _, self.t["wave_noise"] = _timed(pr.mobility, rng.standard_normal(11 * N), 1)
        ori = np.tile([0.0, 0.0, 1.0], (N, 1))
        _, self.t["euler"] = _timed(O.euler_shear, self.pos, ori, np.zeros((N, 4)), rng.standard_normal(6 * N),
                                    np.zeros((N, 3), np.int64), self.L, 0.0, 1e-4, 1.0)
        _, self.t["lanczos_ff_op"] = _timed(pr.mobility, rng.standard_normal(11 * N), 2)
        _, self.t["lanczos_nf_op"] = _timed(pr.rfu, rng.standard_normal(6 * N))
        return self

    def sample_iteration(self, depth: int = 50):
        """One GMRES iteration: saddle operator, preconditioner, Gram-Schmidt at `depth`."""
        N = self.N
        rng = np.random.default_rng(1)
        x = rng.standard_normal(17 * N)
        _, self.t["saddle_op"] = _timed(self.pr.saddle_multiply, x)

        _, self.t["precond_apply"] = _timed(self._pc, x)
        V = rng.standard_normal((depth, 17 * N))
        w = rng.standard_normal(17 * N)

        def cgs2():
            v = w.copy()
            for _ in range(2):
                c = V @ v
                v -= V.T @ c
            return v
        _, self.t["gram_schmidt"] = _timed(cgs2)
        return self

    def _pc(self, b):
        N = self.N
        y = self.ilu.solve(b[: 6 * N] - b[11 * N:])
        out = b.copy()
        out[: 6 * N] = b[: 6 * N] - y
        out[11 * N:] = y
        return out

    def step_seconds(self, iters: dict) -> tuple[float, dict]:
        """Seconds of one step given the IChol method's iteration counts
        (gmres_rfd_plus, gmres_rfd_minus, gmres_main, lanczos_ff, lanczos_nf)."""
        t = self.t
        g = iters["gmres_rfd_plus"] + iters["gmres_rfd_minus"] + iters["gmres_main"]
        per_it = t["saddle_op"] + t["precond_apply"] + t["gram_schmidt"]
        parts = {
            "nlist": t["nlist"], "pair_force": t["pair_force"], "precond_build": t["precond_build"],
            "wave_noise": t["wave_noise"], "lanczos": iters["lanczos_ff"] * t["lanczos_ff_op"]
            + iters["lanczos_nf"] * t["lanczos_nf_op"],
            # each solve also applies the operator for its initial and final true residuals
            "gmres": g * per_it + 6 * t["saddle_op"], "euler": t["euler"],
        }
        return float(sum(parts.values())), parts


def _lanczos_sqrt(op, z, tol=1e-3, max_iter=100):
    """Chow-Saad Lanczos approximation of op^(1/2) z (Brownian_FarField.cu:597-808,
    Brownian_NearField.cu:174-464): m-step Lanczos, square root of the small
    tridiagonal matrix, stopped when the sample changes by less than tol."""
    from scipy.linalg import eigh_tridiagonal
    n = len(z)
    zn = np.linalg.norm(z)
    V = np.zeros((max_iter + 1, n))
    V[0] = z / zn
    alpha, beta = [], []
    prev = None
    y = None
    for m in range(max_iter):
        w = op(V[m])
        if m:
            w -= beta[-1] * V[m - 1]
        a = float(V[m] @ w)
        w -= a * V[m]
        alpha.append(a)
        b = float(np.linalg.norm(w))
        ev, Q = eigh_tridiagonal(np.array(alpha), np.array(beta))
        s = Q @ (np.sqrt(np.maximum(ev, 0.0)) * Q[0])
        y = zn * (V[: m + 1].T @ s)
        if prev is not None and np.linalg.norm(y - prev) <= tol * np.linalg.norm(y):
            return y, m + 1
        prev = y
        if b == 0.0:
            return y, m + 1
        beta.append(b)
        V[m + 1] = w / b
    return y, max_iter


def full_step_seconds(pos, L, table, shear_rate=1.0, kT=1.0, dt=1e-4, tol=1e-4, seed=0):
    """One complete FP64 FSD step with the IChol method's preconditioner
    (SciPy's incomplete LU of the pruned R_FU + D standing in for csric02),
    timed end to end on the host cores: neighbour list, pair force,
    preconditioner build, far-field noise (one wave-space pass for the random
    field plus Lanczos on the real-space mobility), near-field noise (Lanczos
    on R_FU), the two random-finite-difference solves and the main solve
    (GMRES(200) to tol, Saddle.cu:171-264 block preconditioner), stresslet
    and Euler update.  Returns (seconds, stage seconds, iteration counts)."""
    import scipy.sparse.linalg as sla
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    st = StepSampler(pos, L, table)
    N = st.N
    t = {}
    rows, t["nlist"] = _timed(st._neighbor_rows)
    pr = O.Problem(st.pos, st.L, 0.0, table=table, rows=rows)
    F, t["pair_force"] = _timed(O.pair_force, st.pos, st.L, 0.0, rows)

    def build():
        A = O.pruned_rfu_sparse(st.pos, st.L, 0.0, pr.tdist, pr.tvals, rows=rows, rp=2.1).tocsc()
        return sla.spilu(A, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0)
    ilu, t["precond_build"] = _timed(build)
    n = 17 * N

    def pc(b):
        y = ilu.solve(b[: 6 * N] - b[11 * N:])
        x = b.copy()
        x[: 6 * N] = b[: 6 * N] - y
        x[11 * N:] = y
        return x
    Aop = sla.LinearOperator((n, n), matvec=pr.saddle_multiply, dtype=np.float64)
    Mop = sla.LinearOperator((n, n), matvec=pc, dtype=np.float64)
    its = {}

    def solve(rhs, name):
        count = [0]

        def cb(_):
            count[0] += 1
        x, _ = sla.gmres(Aop, rhs, M=Mop, rtol=tol, restart=200, maxiter=20, callback=cb,
                         callback_type="pr_norm")
        its[name] = count[0]
        return x
    scale = np.sqrt(2.0 * kT / dt)
    tb = time.perf_counter()
    wave = pr.mobility(rng.standard_normal(11 * N), 1)
    u_ff, its["lanczos_ff"] = _lanczos_sqrt(lambda v: pr.mobility(v, 2), rng.standard_normal(11 * N))
    f_nf, its["lanczos_nf"] = _lanczos_sqrt(pr.rfu, rng.standard_normal(6 * N))
    t["brownian"] = time.perf_counter() - tb
    tr = time.perf_counter()
    psi = rng.standard_normal(6 * N)
    rhs = np.zeros(n)
    rhs[11 * N:] = -psi
    up = solve(rhs, "gmres_rfd_plus")
    um = solve(rhs, "gmres_rfd_minus")
    t["rfd"] = time.perf_counter() - tr
    tm = time.perf_counter()
    rhs = O.strain_rhs(shear_rate, N)
    rhs[: 11 * N] += scale * (wave + u_ff)
    rhs[11 * N:] += scale * f_nf - F + O.rfe(pr.pos, shear_rate, st.L, 0.0, rows, pr.tdist, pr.tvals)
    x = solve(rhs, "gmres_main")
    U = x[11 * N:] + (kT / 1e-3) * 1e-3 * (up[11 * N:] - um[11 * N:])
    O.rsu(pr.pos, U, st.L, 0.0, rows, pr.tdist, pr.tvals)
    t["main_solve"] = time.perf_counter() - tm
    ori = np.tile([0.0, 0.0, 1.0], (N, 1))
    _, t["euler"] = _timed(O.euler_shear, st.pos, ori, np.zeros((N, 4)), U, np.zeros((N, 3), np.int64), st.L, 0.0,
                           dt, shear_rate)
    return time.perf_counter() - t0, t, its
