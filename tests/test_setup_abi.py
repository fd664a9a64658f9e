"""Host-side product code on CPU: the C ABI loads and exports every entry point
of include/fsd.h, and the PSE set-up (grid, support, splitting, quad-precision
real-space Ewald table) and the RCM ordering equal the reference's."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, golden, rows_from
from fsd_b200 import _lib
from fsd_b200.core import default_params


def header_functions():
    text = (ROOT / "include" / "fsd.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fsd_\w+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = C.CDLL(str(_lib.LIB_PATH))
    names = header_functions()
    assert len(names) >= 28
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.EXPORTED)


def test_status_strings():
    l = _lib.lib()
    assert l.fsd_status_string(0) == b"ok"
    assert b"GMRES" in l.fsd_status_string(3)


def setup(N, L, xi=0.5, error=1e-3, max_strain=0.5, with_table=True):
    p = default_params()
    p.N = N
    p.Lx, p.Ly, p.Lz = L
    p.xi, p.error, p.max_strain = xi, error, max_strain
    info = _lib.fsd_pse_info()
    assert _lib.lib().fsd_pse_setup(C.byref(p), C.byref(info), None, 0) == 0
    tab = None
    if with_table:
        tab = np.zeros((2 * (info.ewald_n + 1), 4), np.float32)
        assert _lib.lib().fsd_pse_setup(C.byref(p), C.byref(info), tab.ctypes.data_as(C.c_void_p), tab.size) == 0
    return info, tab


def test_pse_setup_equals_reference():
    for case in golden("setparams.json"):
        info, _ = setup(100, case["L"], case["xi"], case["error"], case["max_strain"], with_table=False)
        ref = case["ref"]
        assert (info.Nx, info.Ny, info.Nz, info.P) == (ref["Nx"], ref["Ny"], ref["Nz"], ref["P"]), case
        for k in ("ewald_cut", "gauss_m", "eta", "hx", "hy", "hz"):
            assert np.float32(getattr(info, k)) == np.float32(ref[k]), (case, k)


@pytest.mark.parametrize("name,xi,error", [("ewald_xi0.5_err1e-3.npz", 0.5, 1e-3), ("ewald_xi0.8_err1e-4.npz", 0.8, 1e-4)])
def test_ewald_table_bit_identical_to_reference(name, xi, error):
    g = golden(name)
    info, tab = setup(100, (40.0, 40.0, 40.0), xi, error)
    assert info.ewald_n == int(g["n"])
    assert np.float32(info.self_x) == np.float32(g["self_x"]) and np.float32(info.self_y) == np.float32(g["self_y"])
    assert np.array_equal(tab, g["table"])


def test_bad_parameters_are_errors_not_exits():
    p = default_params()
    p.N = 10
    p.Lx = p.Ly = p.Lz = 8.0  # cutoff 5.26 > L/2: the reference exits (Stokes.cc:140-163)
    info = _lib.fsd_pse_info()
    assert _lib.lib().fsd_pse_setup(C.byref(p), C.byref(info), None, 0) == 1


def test_rcm_order_equals_reference():
    p = golden("precond_dense_sheared.npz")
    rows = rows_from(p["pn"], p["pflat"])
    n = len(rows)
    rowptr = np.zeros(n + 1, np.int32)
    rowptr[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int32)
    perm = np.zeros(n, np.int32)
    assert _lib.lib().fsd_rcm_order(n, rowptr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                    perm.ctypes.data_as(C.c_void_p)) == 0
    assert np.array_equal(perm, p["rcm_perm"])
