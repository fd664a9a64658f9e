"""The allocation-free neighbour list against the handle-based one.

fsd_neighbor_list_noalloc exists for callers that cannot allocate device
memory where they need a neighbour list (a host application that owns all
device memory through its own pool, or a step loop that must not call
cudaMalloc/cudaFree because they can synchronise the whole device).  It works
in one fixed device array shared by all calls, so these tests call it twice in
a row on different configurations: a list left over from the first call would
show up in the second.  Lists are integer data, so rows must match the
existing entry point (fsd_build_neighbor_list) exactly as sets.

This file is collected last on purpose, so a run that stops at its first
failure has run every other test before this one.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from fsd_b200 import _lib
from fsd_b200.configs import suspension
from fsd_b200.core import FSD


def _rows(nneigh, nlist, stride):
    return [np.sort(nlist[i * stride: i * stride + nneigh[i]]) for i in range(len(nneigh))]


def _noalloc(pos, L, xy, rlist, stride):
    N = len(pos)
    p = torch.as_tensor(np.ascontiguousarray(pos, np.float32)).cuda().contiguous()
    nneigh = torch.full((N,), 0xFFFF, dtype=torch.int32, device="cuda")
    nlist = torch.full((N * stride,), -1, dtype=torch.int32, device="cuda")
    mx = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    status = _lib.lib().fsd_neighbor_list_noalloc(p.data_ptr(), N, L[0], L[1], L[2], xy, rlist, nneigh.data_ptr(),
                                                  nlist.data_ptr(), stride, mx.data_ptr(), st)
    assert status == 0, _lib.STATUS.get(status)
    torch.cuda.synchronize()
    return nneigh.cpu().numpy().view(np.uint32), nlist.cpu().numpy().view(np.uint32), int(mx.item())


def _handle_rows(pos, L, xy):
    N = len(pos)
    s = FSD(N, (L[0], L[1], L[2], xy))
    p = torch.as_tensor(np.ascontiguousarray(pos, np.float32)).cuda().view(-1).contiguous()
    s.build_neighbor_list(p)
    rows = [np.sort(r) for r in s.neighbor_list()]
    rlist = s.pse_info().ewald_cut + 0.4  # the handle's list radius: Ewald cutoff + default buffer
    nmax = s.solve_info()["nlist_max"]
    s.close()
    return rows, rlist, nmax


@pytest.mark.gpu
def test_noalloc_matches_handle_list_on_two_calls_in_a_row(cuda):
    cases = [suspension(3000, 0.35, 3) + (0.2,),   # cell-list path, sheared box
             suspension(300, 0.3, 5) + (0.0,)]     # box under three cells wide: all-pairs path
    for pos, Lc, xy in cases:
        L = (Lc, Lc, Lc)
        ref, rlist, nmax = _handle_rows(pos, L, xy)
        stride = max(len(r) for r in ref) + 8
        nneigh, nlist, mx = _noalloc(pos, L, xy, rlist, stride)
        assert mx == nmax == max(len(r) for r in ref)
        got = _rows(nneigh, nlist, stride)
        assert all(np.array_equal(a, b) for a, b in zip(got, ref))


@pytest.mark.gpu
def test_noalloc_wider_cells_when_the_cell_grid_exceeds_its_scratch(cuda):
    """A 60-wide box over r_list = 1 would need 60^3 = 216000 cells, more than
    the scratch's 65536: the call falls back to fewer, wider cells, which must
    still give every pair (brute-force sets from the oracle)."""
    from oracle import fsd_oracle as O
    rng = np.random.default_rng(11)
    N, Lc = 4000, 60.0
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = (rng.random((N, 3)) - 0.5) * Lc
    rlist = 1.0
    ref = O.neighbor_list(pos, (Lc, Lc, Lc), 0.0, rlist)
    stride = max(8, max(len(r) for r in ref) + 4)
    for _ in range(2):  # twice in a row: nothing may carry over in the shared scratch
        nneigh, nlist, mx = _noalloc(pos, (Lc, Lc, Lc), 0.0, rlist, stride)
        assert mx == max(len(r) for r in ref)
        got = _rows(nneigh, nlist, stride)
        assert all(np.array_equal(a, np.sort(b)) for a, b in zip(got, ref))


@pytest.mark.gpu
def test_noalloc_reports_truncated_rows(cuda):
    pos, Lc = suspension(2000, 0.3, 7)
    L = (Lc, Lc, Lc)
    ref, rlist, nmax = _handle_rows(pos, L, 0.0)
    stride = 16
    nneigh, nlist, mx = _noalloc(pos, L, 0.0, rlist, stride)
    assert mx == nmax > stride
    assert np.array_equal(nneigh, np.minimum([len(r) for r in ref], stride))
    for i, r in enumerate(ref):  # kept entries are true neighbours
        assert set(nlist[i * stride: i * stride + nneigh[i]]) <= set(r)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    """Rejected on the host before any GPU work, so this runs without a GPU."""
    lib = _lib.lib()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    too_many = 65536 + 1
    assert lib.fsd_neighbor_list_noalloc(dummy, too_many, 50.0, 50.0, 50.0, 0.0, 5.0, dummy, dummy, 64, dummy,
                                         None) == 1
    assert lib.fsd_neighbor_list_noalloc(dummy, 100, 50.0, 50.0, 50.0, 0.0, 5.0, dummy, dummy, 0, dummy, None) == 1
    assert lib.fsd_neighbor_list_noalloc(dummy, 100, -1.0, 50.0, 50.0, 0.0, 5.0, dummy, dummy, 64, dummy, None) == 1
    assert lib.fsd_neighbor_list_noalloc(None, 100, 50.0, 50.0, 50.0, 0.0, 5.0, dummy, dummy, 64, dummy, None) == 1
