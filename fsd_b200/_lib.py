"""ctypes binding of the C ABI in include/fsd.h (libfsd.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback
for any operator of this package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfsd.so"

FSD_OK = 0
REGIONS = ("nlist", "precond_build", "spread", "fft", "green", "contract", "real_space", "rfu", "precond_apply",
           "krylov", "lanczos", "brownian_wave", "lub_other", "integrate")
STATUS = {
    0: "FSD_OK", 1: "FSD_ERR_BAD_PARAMS", 2: "FSD_ERR_CUDA", 3: "FSD_ERR_GMRES_MAXIT",
    4: "FSD_ERR_LANCZOS_MAXIT", 5: "FSD_ERR_ICHOL", 6: "FSD_ERR_NLIST_OVERFLOW",
    7: "FSD_ERR_DEVICE_WAIT", 8: "FSD_ERR_ALLOC", 9: "FSD_ERR_BREAKDOWN",
}
PRECOND = {"none": 0, "ichol": 1, "learned": 2}
FORCE_MODE = {"interparticle": 0, "user": 1}


class fsd_params(C.Structure):
    _fields_ = [
        ("N", C.c_int),
        ("Lx", C.c_float), ("Ly", C.c_float), ("Lz", C.c_float), ("xy", C.c_float),
        ("xi", C.c_float), ("error", C.c_float), ("max_strain", C.c_float),
        ("solver_tol", C.c_float), ("lanczos_tol", C.c_float), ("rfd_epsilon", C.c_float),
        ("T", C.c_float), ("dt", C.c_float), ("seed", C.c_uint32),
        ("ndsr", C.c_float), ("kappa", C.c_float), ("k_n", C.c_float), ("beta_AF", C.c_float), ("epsq", C.c_float),
        ("T_ext", C.c_float), ("omega_ext", C.c_float),
        ("sqm_B1", C.c_float), ("sqm_B2", C.c_float),
        ("N_mix", C.c_int), ("coef_B1_mask", C.c_float), ("coef_B2_mask", C.c_float),
        ("rot_diff", C.c_float),
        ("period", C.c_int),
        ("gmres_restart", C.c_int), ("gmres_max_iter", C.c_int), ("lanczos_max", C.c_int),
        ("precond", C.c_int), ("force_mode", C.c_int), ("kgrid_pi_ref", C.c_int),
        ("rlub", C.c_float), ("rp", C.c_float), ("nlist_buffer", C.c_float),
        ("ichol_local_shift", C.c_int), ("ichol_gain_limit", C.c_float),
        ("learned_inner", C.c_int), ("learned_poly", C.c_int), ("poly_interval", C.c_float), ("autotune", C.c_int),
        ("friction_type", C.c_int), ("friction_h0", C.c_float), ("friction_alpha", C.c_float * 6),
        ("integrator", C.c_int),
    ]


class fsd_pse_info(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("P", C.c_int),
        ("ewald_cut", C.c_float), ("gauss_m", C.c_float), ("eta", C.c_float),
        ("hx", C.c_float), ("hy", C.c_float), ("hz", C.c_float),
        ("self_x", C.c_float), ("self_y", C.c_float),
        ("ewald_n", C.c_int), ("ewald_dr", C.c_float),
    ]


class fsd_solve_info(C.Structure):
    _fields_ = [
        ("gmres_iters", C.c_int * 3), ("gmres_resid", C.c_float * 3),
        ("lanczos_ff_iters", C.c_int), ("lanczos_nf_iters", C.c_int),
        ("lanczos_ff_err", C.c_float), ("lanczos_nf_err", C.c_float),
        ("ichol_attempts", C.c_int), ("ichol_relaxer", C.c_float),
        ("nlist_max", C.c_int), ("status", C.c_int), ("ichol_shifted", C.c_int),
        ("ichol_gain", C.c_float),
        ("poly_source", C.c_int), ("poly_loss_net", C.c_float), ("poly_loss_fit", C.c_float),
        ("poly_ratio", C.c_float),
    ]


class fsd_step_args(C.Structure):
    _fields_ = [
        ("timestep", C.c_uint), ("shear_rate", C.c_float),
        ("d_pos", C.c_void_p), ("d_ori", C.c_void_p), ("d_pos_gb", C.c_void_p), ("d_image", C.c_void_p),
        ("d_force", C.c_void_p), ("d_velocity", C.c_void_p), ("d_noise_ang", C.c_void_p),
        ("d_b1_mask", C.c_void_p), ("d_b2_mask", C.c_void_p),
    ]


H = C.c_void_p
P = C.c_void_p
_SIGS = {
    "fsd_default_params": (None, [C.POINTER(fsd_params)]),
    "fsd_status_string": (C.c_char_p, [C.c_int]),
    "fsd_pse_setup": (C.c_int, [C.POINTER(fsd_params), C.POINTER(fsd_pse_info), P, C.c_size_t]),
    "fsd_rcm_order": (C.c_int, [C.c_int, P, P, P]),
    "fsd_resistance_table": (C.c_int, [C.POINTER(fsd_params), P, P]),
    "fsd_create": (C.c_int, [C.POINTER(fsd_params), P, C.POINTER(H)]),
    "fsd_destroy": (None, [H]),
    "fsd_set_stream": (C.c_int, [H, P]),
    "fsd_launch_count": (C.c_ulonglong, []),
    "fsd_set_box": (C.c_int, [H, C.c_float, C.c_float, C.c_float, C.c_float]),
    "fsd_set_temperature": (C.c_int, [H, C.c_float]),
    "fsd_get_pse_info": (C.c_int, [H, C.POINTER(fsd_pse_info)]),
    "fsd_get_solve_info": (C.c_int, [H, C.POINTER(fsd_solve_info)]),
    "fsd_checkpoint_size": (C.c_size_t, [H]),
    "fsd_checkpoint_save": (C.c_int, [H, P, C.c_size_t]),
    "fsd_checkpoint_load": (C.c_int, [H, P, C.c_size_t]),
    "fsd_profile_enable": (C.c_int, [H, C.c_int]),
    "fsd_profile_read": (C.c_int, [H, P, P, C.c_int, C.c_int]),
    "fsd_get_ewald_table": (C.c_int, [H, P, C.c_size_t]),
    "fsd_build_neighbor_list": (C.c_int, [H, P]),
    "fsd_get_neighbor_list": (C.c_int, [H, P, P, C.c_size_t, C.POINTER(C.c_int)]),
    "fsd_neighbor_list_noalloc": (C.c_int, [P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                            P, P, C.c_int, P, P]),
    "fsd_mobility": (C.c_int, [H, P, P, P, C.c_int]),
    "fsd_lub_rfu": (C.c_int, [H, P, P, P]),
    "fsd_lub_rfe": (C.c_int, [H, P, C.c_float, P, P, C.c_float, P]),
    "fsd_lub_rsu": (C.c_int, [H, P, P, P]),
    "fsd_lub_rse": (C.c_int, [H, P, C.c_float, P, P, C.c_float, P]),
    "fsd_saddle_multiply": (C.c_int, [H, P, P, P]),
    "fsd_precond_build": (C.c_int, [H, P]),
    "fsd_precond_set_blocks": (C.c_int, [H, C.c_int, P, P, P]),
    "fsd_learned_num_weights": (C.c_int, []),
    "fsd_learned_set_weights": (C.c_int, [H, P, C.c_int]),
    "fsd_learned_get_weights": (C.c_int, [H, P, C.c_int]),
    "fsd_learned_tensor_cores": (C.c_int, [H, C.c_int]),
    "fsd_learned_get_state": (C.c_int, [H, P, C.c_int, C.POINTER(C.c_int)]),
    "fsd_learned_set_state": (C.c_int, [H, P, C.c_int, C.c_int]),
    "fsd_learned_train_step": (C.c_int, [H, P, P, C.c_int, C.c_uint, C.c_float, C.POINTER(C.c_float), P]),
    "fsd_learned_set_poly": (C.c_int, [H, P, C.c_int]),
    "fsd_learned_get_poly": (C.c_int, [H, P, C.c_int]),
    "fsd_learned_set_interval": (C.c_int, [H, C.c_float]),
    "fsd_learned_interval_coefficients": (C.c_int, [C.c_float, C.c_float, C.c_int, P]),
    "fsd_learned_ratio_train_step": (C.c_int, [H, P, C.c_float, C.c_float, C.POINTER(C.c_float),
                                               C.POINTER(C.c_float), P]),
    "fsd_learned_poly_train_step": (C.c_int, [H, P, C.c_int, C.c_uint, C.c_float, C.c_int, C.POINTER(C.c_float),
                                              C.POINTER(C.c_float), P, P, P]),
    "fsd_precond_apply": (C.c_int, [H, P, P]),
    "fsd_saddle_solve": (C.c_int, [H, P, P, P, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "fsd_brownian_farfield": (C.c_int, [H, P, C.c_uint, P]),
    "fsd_brownian_nearfield": (C.c_int, [H, P, C.c_uint, P]),
    "fsd_rfd_drift": (C.c_int, [H, P, P, C.c_uint, P]),
    "fsd_draw_normals": (C.c_int, [H, C.c_uint, C.c_uint, C.c_size_t, C.c_float, P]),
    "fsd_integrate_euler": (C.c_int, [H, C.POINTER(fsd_step_args)]),
    "fsd_compute_velocity": (C.c_int, [H, C.POINTER(fsd_step_args)]),
    "fsd_step": (C.c_int, [H, C.POINTER(fsd_step_args)]),
    "fsd_step_batch": (C.c_int, [P, P, C.c_int, C.c_int, P]),
}
EXPORTED = tuple(_SIGS)

_lib = None


class FSDError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)} ({lib().fsd_status_string(status).decode()})")


def lib():
    """The loaded libfsd.so with typed signatures; raises if it is absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m fsd_b200.build`")
        l = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(status: int, what: str) -> int:
    if status != FSD_OK:
        raise FSDError(status, what)
    return status
