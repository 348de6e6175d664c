"""The allocation-free MSI entry point (m2d_msi_solve_device_noalloc).

Callers whose device memory is all owned by their own pool, or whose hot loop
must not call cudaMalloc/cudaFree (both synchronise the device), use this
variant: its workspace is a fixed 12 MiB array inside the library, found with
cudaGetSymbolAddress on the first call on each device.  The test calls it
through the C ABI twice in a row, on two different systems, and checks each
result against the allocating entry point (m2d_msi_solve_device with a
caller-provided workspace) with the same bitwise bar as the other solver
tests; it also checks the size limit.  This file is collected last so that a
run stopping at the first failure has already run every other test; it
passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

from _systems import dirichlet_system, random_dominant_planes
from mach2d_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def _bind():
    L = lib()
    L.m2d_msi_workspace_doubles.restype = ctypes.c_long
    L.m2d_msi_workspace_doubles.argtypes = [ctypes.c_int] * 3
    L.m2d_msi_noalloc_max_cells.restype = ctypes.c_long
    L.m2d_msi_noalloc_max_cells.argtypes = [ctypes.c_int]
    L.m2d_msi_solve_device.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
    L.m2d_msi_solve_device_noalloc.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 5
    return L


def _solve_both(L, nd, nx, ny, nitm, tol, a, b):
    import torch
    dev = torch.device("cuda:0")
    N = nx * ny
    da = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    work = torch.empty(L.m2d_msi_workspace_doubles(nd, nx, ny), dtype=torch.float64, device=dev)
    x_ref = torch.zeros(N, dtype=torch.float64, device=dev)
    x_new = torch.zeros(N, dtype=torch.float64, device=dev)
    nit = torch.zeros(2, dtype=torch.int32, device=dev)
    check(L.m2d_msi_solve_device(nd, nx, ny, nitm, tol, da.data_ptr(), db.data_ptr(), x_ref.data_ptr(),
                                 work.data_ptr(), None, nit.data_ptr()))
    check(L.m2d_msi_solve_device_noalloc(nd, nx, ny, nitm, tol, da.data_ptr(), db.data_ptr(),
                                         x_new.data_ptr(), None, nit.data_ptr() + 4))
    torch.cuda.synchronize()
    return x_ref.cpu().numpy(), x_new.cpu().numpy(), nit.cpu().numpy()


@pytest.mark.parametrize("nd", [9, 5])
def test_noalloc_one_cta_fallback_matches_allocating_entry_point(nd):
    # 400 x 300 is under the cell limit, but its wavefront-major layout
    # (21 or 15 planes of 320 x 462) does not fit in the array, so the
    # noalloc call runs the one-CTA kernel while the allocating call, with a
    # full workspace, runs the cluster kernel; the two are bitwise equal
    L = _bind()
    nx, ny = 400, 300
    assert nx * ny <= L.m2d_msi_noalloc_max_cells(nd)
    a, b = dirichlet_system(nd, nx, ny, seed=33)
    x_ref, x_new, nit = _solve_both(L, nd, nx, ny, 5, 1e-6, a, b)
    assert nit[0] == nit[1] and nit[0] >= 1
    assert np.array_equal(x_ref, x_new)


@pytest.mark.parametrize("nd", [9, 5])
def test_noalloc_solve_matches_allocating_entry_point_twice(nd):
    L = _bind()
    # two calls in a row on the shared scratch, different sizes and systems
    systems = [(258, 130, 20, 1e-8, dirichlet_system(nd, 258, 130, seed=31)),
               (97, 45, 5, 1e-2, random_dominant_planes(nd, 97, 45, seed=32))]
    for nx, ny, nitm, tol, (a, b) in systems:
        x_ref, x_new, nit = _solve_both(L, nd, nx, ny, nitm, tol, a, b)
        assert nit[0] == nit[1] and nit[0] >= 1
        assert np.array_equal(x_ref, x_new)


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = _bind()
    limit = L.m2d_msi_noalloc_max_cells(9)
    assert limit == 157286 and L.m2d_msi_noalloc_max_cells(5) == 196607
    nx, ny = 400, 400                                   # 160000 cells > 157286
    buf = ctypes.c_void_p(1)                            # never dereferenced: the size check comes first
    rc = L.m2d_msi_solve_device_noalloc(9, nx, ny, 5, 1e-2, buf, buf, buf, None, None)
    assert rc == 6
    assert b"maximum" in L.m2d_last_error()
