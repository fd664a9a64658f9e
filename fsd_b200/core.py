"""Operator-level handle over the C ABI, on torch CUDA tensors.

``FSD`` owns one ``fsd_handle`` (device tables, workspaces, preconditioner)
and exposes each piece of the velocity path on device tensors in the
reference's layouts (positions float4, generalized 11N vectors, saddle 17N
vectors).  torch is used only for device memory and the current stream.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check, lib


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor expected")
    return t.data_ptr()


def _f32(t: torch.Tensor, n: int, what: str) -> torch.Tensor:
    if t.dtype != torch.float32 or t.numel() != n:
        raise ValueError(f"{what}: float32 tensor with {n} elements expected, got {t.dtype} {tuple(t.shape)}")
    return t


@dataclass
class PSEInfo:
    Nx: int
    Ny: int
    Nz: int
    P: int
    ewald_cut: float
    gauss_m: float
    eta: float
    hx: float
    hy: float
    hz: float
    self_x: float
    self_y: float
    ewald_n: int
    ewald_dr: float


def default_params() -> _lib.fsd_params:
    p = _lib.fsd_params()
    lib().fsd_default_params(C.byref(p))
    return p


class FSD:
    """One suspension of N unit spheres in a periodic (optionally sheared) box."""

    def __init__(self, N: int, box, device: str | torch.device = "cuda", **kw):
        p = default_params()
        p.N = int(N)
        Lx, Ly, Lz = box[:3]
        p.Lx, p.Ly, p.Lz = float(Lx), float(Ly), float(Lz)
        p.xy = float(box[3]) if len(box) > 3 else 0.0
        for k, v in kw.items():
            if k == "precond":
                v = _lib.PRECOND[v] if isinstance(v, str) else int(v)
            elif k == "force_mode":
                v = _lib.FORCE_MODE[v] if isinstance(v, str) else int(v)
            elif k == "friction_alpha" and not isinstance(v, C.Array):
                v = (C.c_float * 6)(*[float(a) for a in v])
            elif k == "friction_type" and isinstance(v, str):
                v = {"NONE": 0, "TYPE1": 1}[v.upper()]
            elif k == "integrator" and isinstance(v, str):
                v = {"euler": 0, "rk2": 1}[v.lower()]
            if not hasattr(p, k):
                raise TypeError(f"unknown parameter {k}")
            setattr(p, k, v)
        self.params = p
        self.N = p.N
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("the FSD velocity path runs on CUDA devices only")
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            check(lib().fsd_create(C.byref(p), C.c_void_p(stream), C.byref(self._h)), "fsd_create")

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if self._h:
            lib().fsd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sync_stream(self):
        stream = torch.cuda.current_stream(self.device).cuda_stream
        check(lib().fsd_set_stream(self._h, C.c_void_p(stream)), "fsd_set_stream")

    # -- info ----------------------------------------------------------------
    def pse_info(self) -> PSEInfo:
        info = _lib.fsd_pse_info()
        check(lib().fsd_get_pse_info(self._h, C.byref(info)), "fsd_get_pse_info")
        return PSEInfo(*[getattr(info, f) for f, _ in info._fields_])

    def checkpoint(self) -> bytes:
        """The solver state this handle carries into the next step (warm start,
        Lanczos sizes, IC(0) relaxer), as bytes for fsd_checkpoint_load."""
        self._sync_stream()
        n = lib().fsd_checkpoint_size(self._h)
        buf = C.create_string_buffer(n)
        check(lib().fsd_checkpoint_save(self._h, buf, n), "fsd_checkpoint_save")
        return buf.raw

    def restore(self, data: bytes):
        """Load a checkpoint written by checkpoint() on a handle of the same N."""
        self._sync_stream()
        buf = C.create_string_buffer(bytes(data), len(data))
        check(lib().fsd_checkpoint_load(self._h, buf, len(data)), "fsd_checkpoint_load")

    def solve_info(self) -> dict:
        info = _lib.fsd_solve_info()
        check(lib().fsd_get_solve_info(self._h, C.byref(info)), "fsd_get_solve_info")
        out = {f: getattr(info, f) for f, _ in info._fields_}
        out["gmres_iters"] = list(info.gmres_iters)
        out["gmres_resid"] = list(info.gmres_resid)
        return out

    def ewald_table(self) -> np.ndarray:
        n = self.pse_info().ewald_n + 1
        out = np.zeros((2 * n, 4), np.float32)
        check(lib().fsd_get_ewald_table(self._h, out.ctypes.data_as(C.c_void_p), out.size), "fsd_get_ewald_table")
        return out

    def set_box(self, Lx, Ly, Lz, xy):
        check(lib().fsd_set_box(self._h, Lx, Ly, Lz, xy), "fsd_set_box")
        self.params.xy = float(xy)

    def set_temperature(self, T):
        check(lib().fsd_set_temperature(self._h, T), "fsd_set_temperature")
        self.params.T = float(T)

    # -- neighbour list --------------------------------------------------------
    def build_neighbor_list(self, pos: torch.Tensor):
        self._sync_stream()
        _f32(pos, 4 * self.N, "pos")
        check(lib().fsd_build_neighbor_list(self._h, _ptr(pos)), "fsd_build_neighbor_list")

    def neighbor_list(self) -> list[np.ndarray]:
        stride = C.c_int()
        nn = np.zeros(self.N, np.uint32)
        check(lib().fsd_get_neighbor_list(self._h, nn.ctypes.data_as(C.c_void_p), None, 0, C.byref(stride)),
              "fsd_get_neighbor_list")
        rows = np.zeros((self.N, stride.value), np.uint32)
        check(lib().fsd_get_neighbor_list(self._h, None, rows.ctypes.data_as(C.c_void_p), rows.size, C.byref(stride)),
              "fsd_get_neighbor_list")
        return [rows[i, : nn[i]].copy() for i in range(self.N)]

    # -- operators -------------------------------------------------------------
    def _new(self, n):
        return torch.zeros(n, dtype=torch.float32, device=self.device)

    def mobility(self, pos, genF, parts: int = 3) -> torch.Tensor:
        self._sync_stream()
        _f32(genF, 11 * self.N, "genF")
        out = self._new(11 * self.N)
        check(lib().fsd_mobility(self._h, _ptr(pos), _ptr(genF), _ptr(out), parts), "fsd_mobility")
        return out

    def rfu(self, pos, U) -> torch.Tensor:
        self._sync_stream()
        _f32(U, 6 * self.N, "U")
        out = self._new(6 * self.N)
        check(lib().fsd_lub_rfu(self._h, _ptr(pos), _ptr(U), _ptr(out)), "fsd_lub_rfu")
        return out

    def rfe(self, pos, shear_rate, ori=None, b2_mask=None, B2=0.0, out=None) -> torch.Tensor:
        self._sync_stream()
        out = self._new(6 * self.N) if out is None else out
        check(lib().fsd_lub_rfe(self._h, _ptr(pos), shear_rate, _ptr(ori), _ptr(b2_mask), B2, _ptr(out)),
              "fsd_lub_rfe")
        return out

    def rsu(self, pos, U, out=None) -> torch.Tensor:
        self._sync_stream()
        out = self._new(5 * self.N) if out is None else out
        check(lib().fsd_lub_rsu(self._h, _ptr(pos), _ptr(U), _ptr(out)), "fsd_lub_rsu")
        return out

    def rse(self, pos, shear_rate, ori=None, b2_mask=None, B2=0.0, out=None) -> torch.Tensor:
        self._sync_stream()
        out = self._new(5 * self.N) if out is None else out
        check(lib().fsd_lub_rse(self._h, _ptr(pos), shear_rate, _ptr(ori), _ptr(b2_mask), B2, _ptr(out)),
              "fsd_lub_rse")
        return out

    def saddle_multiply(self, pos, x) -> torch.Tensor:
        self._sync_stream()
        _f32(x, 17 * self.N, "x")
        out = self._new(17 * self.N)
        check(lib().fsd_saddle_multiply(self._h, _ptr(pos), _ptr(x), _ptr(out)), "fsd_saddle_multiply")
        return out

    def precond_build(self, pos):
        self._sync_stream()
        check(lib().fsd_precond_build(self._h, _ptr(pos)), "fsd_precond_build")

    def precond_set_blocks(self, rowptr, col, blocks):
        """Block-CSR G (int32 rowptr N+1, int32 col, float32 blocks nnzb x 36) for precond='learned'."""
        self._sync_stream()
        rowptr = torch.as_tensor(rowptr, dtype=torch.int32, device=self.device).contiguous()
        col = torch.as_tensor(col, dtype=torch.int32, device=self.device).contiguous()
        blocks = torch.as_tensor(blocks, dtype=torch.float32, device=self.device).contiguous()
        check(lib().fsd_precond_set_blocks(self._h, int(col.numel()), _ptr(rowptr), _ptr(col), _ptr(blocks)),
              "fsd_precond_set_blocks")
        torch.cuda.synchronize(self.device)

    def learned_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        check(lib().fsd_learned_set_weights(self._h, w.ctypes.data_as(C.c_void_p), int(w.size)),
              "fsd_learned_set_weights")

    def learned_get_weights(self) -> np.ndarray:
        w = np.zeros(lib().fsd_learned_num_weights(), np.float32)
        check(lib().fsd_learned_get_weights(self._h, w.ctypes.data_as(C.c_void_p), int(w.size)),
              "fsd_learned_get_weights")
        return w

    def learned_get_state(self):
        n = 3 * lib().fsd_learned_num_weights()
        buf = np.zeros(n, np.float32)
        t = C.c_int(0)
        check(lib().fsd_learned_get_state(self._h, buf.ctypes.data_as(C.c_void_p), n, C.byref(t)),
              "fsd_learned_get_state")
        return buf, t.value

    def learned_set_state(self, state):
        buf, t = state
        buf = np.ascontiguousarray(buf, np.float32)
        check(lib().fsd_learned_set_state(self._h, buf.ctypes.data_as(C.c_void_p), int(buf.size), int(t)),
              "fsd_learned_set_state")

    def learned_set_poly(self, coef):
        """Fixed Chebyshev coefficients of the inner polynomial (learned_poly mode)."""
        c = np.ascontiguousarray(coef, np.float32)
        check(lib().fsd_learned_set_poly(self._h, c.ctypes.data_as(C.c_void_p), int(c.size)), "fsd_learned_set_poly")

    def learned_get_poly(self):
        """(coefficients in use, spectral bound lambda of AG of the last build)."""
        buf = np.zeros(17, np.float32)
        check(lib().fsd_learned_get_poly(self._h, buf.ctypes.data_as(C.c_void_p), 17), "fsd_learned_get_poly")
        k = self.params.learned_poly
        return buf[:k].copy(), float(buf[16])

    def learned_poly_train_step(self, pos, n_probes=4, step=0, lr=0.0, want_grad=False, natural=False):
        """Inner-polynomial loss of this configuration with the network's
        coefficients, its least-squares optimum, both coefficient sets, the
        weight gradient (when want_grad) and, for lr > 0, one Adam step."""
        self._sync_stream()
        k = self.params.learned_poly
        loss, loss_opt = C.c_float(0.0), C.c_float(0.0)
        coef, copt = np.zeros(k, np.float32), np.zeros(k, np.float32)
        g = np.zeros(lib().fsd_learned_num_weights(), np.float32) if want_grad else None
        check(lib().fsd_learned_poly_train_step(self._h, _ptr(pos), int(n_probes), int(step), float(lr),
                                                int(bool(natural)), C.byref(loss), C.byref(loss_opt),
                                                g.ctypes.data_as(C.c_void_p) if want_grad else None,
                                                coef.ctypes.data_as(C.c_void_p), copt.ctypes.data_as(C.c_void_p)),
              "fsd_learned_poly_train_step")
        out = {"loss": loss.value, "loss_opt": loss_opt.value, "coef": coef, "coef_opt": copt}
        if want_grad:
            out["grad"] = g
        return out

    def learned_set_interval(self, rho: float):
        """Fixed Chebyshev interval ratio for the next builds (0 clears it)."""
        check(lib().fsd_learned_set_interval(self._h, float(rho)), "fsd_learned_set_interval")

    def learned_ratio_train_step(self, pos, target_log_ratio: float, lr: float = 0.0, want_grad: bool = False):
        """(squared error, predicted log ratio[, weight gradient]) of the interval network on this configuration."""
        self._sync_stream()
        loss, pred = C.c_float(0.0), C.c_float(0.0)
        g = np.zeros(lib().fsd_learned_num_weights(), np.float32) if want_grad else None
        check(lib().fsd_learned_ratio_train_step(self._h, _ptr(pos), float(target_log_ratio), float(lr),
                                                 C.byref(loss), C.byref(pred),
                                                 g.ctypes.data_as(C.c_void_p) if want_grad else None),
              "fsd_learned_ratio_train_step")
        return (loss.value, pred.value, g) if want_grad else (loss.value, pred.value)

    def learned_tensor_cores(self, on: bool):
        check(lib().fsd_learned_tensor_cores(self._h, int(bool(on))), "fsd_learned_tensor_cores")

    def learned_train_step(self, pos, probes=None, n_probes=4, step=0, lr=0.0, want_grad=False):
        """Loss (and gradient as a NumPy vector when want_grad) of the approximate-inverse
        objective for these positions; lr > 0 also takes one Adam step."""
        self._sync_stream()
        pp = None
        if probes is not None:
            probes = np.ascontiguousarray(probes, np.float32)
            n_probes = probes.shape[0]
            pp = probes.ctypes.data_as(C.c_void_p)
        loss = C.c_float(0.0)
        g = np.zeros(lib().fsd_learned_num_weights(), np.float32) if want_grad else None
        check(lib().fsd_learned_train_step(self._h, _ptr(pos), pp, int(n_probes), int(step), float(lr),
                                           C.byref(loss), g.ctypes.data_as(C.c_void_p) if want_grad else None),
              "fsd_learned_train_step")
        return (loss.value, g) if want_grad else loss.value

    def precond_apply(self, b) -> torch.Tensor:
        self._sync_stream()
        out = self._new(17 * self.N)
        check(lib().fsd_precond_apply(self._h, _ptr(b), _ptr(out)), "fsd_precond_apply")
        return out

    def saddle_solve(self, pos, rhs, x0=None, raise_on_error=True):
        self._sync_stream()
        x = self._new(17 * self.N) if x0 is None else x0.clone()
        it = C.c_int()
        res = C.c_float()
        st = lib().fsd_saddle_solve(self._h, _ptr(pos), _ptr(rhs), _ptr(x), C.byref(it), C.byref(res))
        if raise_on_error:
            check(st, "fsd_saddle_solve")
        return x, it.value, res.value, st

    def brownian_farfield(self, pos, timestep: int) -> torch.Tensor:
        self._sync_stream()
        out = self._new(11 * self.N)
        check(lib().fsd_brownian_farfield(self._h, _ptr(pos), timestep, _ptr(out)), "fsd_brownian_farfield")
        return out

    def brownian_nearfield(self, pos, timestep: int) -> torch.Tensor:
        self._sync_stream()
        out = self._new(6 * self.N)
        check(lib().fsd_brownian_nearfield(self._h, _ptr(pos), timestep, _ptr(out)), "fsd_brownian_nearfield")
        return out

    def rfd_drift(self, pos, image, timestep: int) -> torch.Tensor:
        self._sync_stream()
        out = self._new(6 * self.N)
        check(lib().fsd_rfd_drift(self._h, _ptr(pos), _ptr(image), timestep, _ptr(out)), "fsd_rfd_drift")
        return out

    def draw_normals(self, stream_id: int, timestep: int, n: int, scale: float = 1.0) -> torch.Tensor:
        """The library's counter-based normals of one random stream (fsd_draw_normals)."""
        self._sync_stream()
        out = self._new(n)
        check(lib().fsd_draw_normals(self._h, int(stream_id), int(timestep), int(n), float(scale), _ptr(out)),
              "fsd_draw_normals")
        return out

    def integrate_euler(self, timestep, shear_rate, pos, ori, image, velocity, pos_gb=None, noise_ang=None,
                        b1_mask=None):
        """Euler + shear update from the velocity in `velocity` (fsd_integrate_euler)."""
        self._sync_stream()
        a = self._args(timestep, shear_rate, pos, ori, pos_gb, image, None, velocity, noise_ang, b1_mask, None)
        return check(lib().fsd_integrate_euler(self._h, C.byref(a)), "fsd_integrate_euler")

    def step_args(self, timestep, shear_rate, pos, ori, image, force, velocity, pos_gb=None, noise_ang=None,
                  b1_mask=None, b2_mask=None):
        return self._args(timestep, shear_rate, pos, ori, pos_gb, image, force, velocity, noise_ang, b1_mask, b2_mask)

    def _args(self, timestep, shear_rate, pos, ori, pos_gb, image, force, velocity, noise_ang, b1_mask, b2_mask):
        a = _lib.fsd_step_args()
        a.timestep = int(timestep)
        a.shear_rate = float(shear_rate)
        a.d_pos, a.d_ori, a.d_pos_gb, a.d_image = _ptr(pos), _ptr(ori), _ptr(pos_gb), _ptr(image)
        a.d_force, a.d_velocity = _ptr(force), _ptr(velocity)
        a.d_noise_ang, a.d_b1_mask, a.d_b2_mask = _ptr(noise_ang), _ptr(b1_mask), _ptr(b2_mask)
        return a

    def compute_velocity(self, timestep, shear_rate, pos, ori, image, force, velocity, pos_gb=None, noise_ang=None,
                         b1_mask=None, b2_mask=None) -> int:
        self._sync_stream()
        a = self._args(timestep, shear_rate, pos, ori, pos_gb, image, force, velocity, noise_ang, b1_mask, b2_mask)
        return check(lib().fsd_compute_velocity(self._h, C.byref(a)), "fsd_compute_velocity")

    def step(self, timestep, shear_rate, pos, ori, image, force, velocity, pos_gb=None, noise_ang=None, b1_mask=None,
             b2_mask=None, raise_on_error=True) -> int:
        self._sync_stream()
        a = self._args(timestep, shear_rate, pos, ori, pos_gb, image, force, velocity, noise_ang, b1_mask, b2_mask)
        st = lib().fsd_step(self._h, C.byref(a))
        if raise_on_error:
            check(st, "fsd_step")
        return st


def step_batch(solvers, args, nthreads: int = 0, raise_on_error: bool = True):
    """One step of each solver concurrently (fsd_step_batch); args from FSD.step_args.
    Solvers should live on distinct CUDA streams for their kernels to overlap."""
    n = len(solvers)
    hs = (C.c_void_p * n)(*[s._h.value for s in solvers])
    arr = (_lib.fsd_step_args * n)(*args)
    st = (C.c_int * n)()
    first = lib().fsd_step_batch(C.cast(hs, C.c_void_p), C.cast(arr, C.c_void_p), n, int(nthreads),
                                 C.cast(st, C.c_void_p))
    if raise_on_error:
        check(first, "fsd_step_batch")
    return list(st)
