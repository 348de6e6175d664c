"""Parity of the MSI and line-TDMA kernels with the oracle's lexicographic
restatement of the reference solvers.

The wavefront MSI kernel evaluates every factor and sweep value with the
reference's expression and operand order, so x must be bitwise equal when
both stop after the same number of iterations (the stopping test's sum of
squares is accumulated in a different order; the iteration counts are
checked equal).  Failure paths are exercised without faulting the GPU: a
zero pivot is reported through the status code, and an unbounded iteration
(nitm <= 0) that cannot converge ends at its cap with M2D_ERR_TIMEOUT.
"""
import ctypes

import numpy as np
import pytest

from _oracle import call as orc
from _systems import dirichlet_system, random_dominant_planes, tdma_lines_system
from mach2d_b200 import M2DError
from mach2d_b200._lib import call
from mach2d_b200.solvers import (ClassSolverMSI5d, ClassSolverMSI9d, ClassSolverTDMA5d,
                                 ClassSolverTDMA9d, norm_l1_5d, norm_l1_9d, norm_l1_9d_relative,
                                 tdma_lines)

pytestmark = pytest.mark.gpu


def _gpu_msi(nd, nx, ny, nitm, tol, a, b, x):
    s = (ClassSolverMSI9d if nd == 9 else ClassSolverMSI5d)().init(nx, ny, nitm, tol)
    s.solve(a, b, x)
    return s.nit


@pytest.mark.parametrize("nd", [9, 5])
@pytest.mark.parametrize("nx,ny,nitm,tol,seed", [
    (7, 5, 5, 1e-2, 0),          # smallest grids: every cell is a special case
    (33, 17, 5, 1e-2, 1),
    (66, 34, 20, 1e-2, 2),
    (130, 70, 30, 1e-6, 3),
    (40, 300, 4, 1e-30, 4),      # ny > nx: long wavefront, several rows per thread pass
    # 2^16 cells and more: the residual passes run on the whole GPU and a
    # continuation launch iterates; stopped by the tolerance, by a cap of
    # one iteration (the first launch's state alone) and of two
    (300, 240, 40, 1e-8, 5),
    (260, 256, 1, 1e-30, 6),
    (260, 256, 2, 1e-30, 7),
])
def test_msi_bitwise(nd, nx, ny, nitm, tol, seed):
    a, b = random_dominant_planes(nd, nx, ny, seed=seed)
    x0 = np.random.default_rng(seed + 100).standard_normal(nx * ny)
    xg, xo = x0.copy(), x0.copy()
    nit_g = _gpu_msi(nd, nx, ny, nitm, tol, a, b, xg)
    nit_o = orc(f"msi{nd}_solve", nx, ny, nitm, tol, a, b, xo)
    assert nit_g == nit_o
    assert np.array_equal(xg, xo), np.max(np.abs(xg - xo))


@pytest.mark.parametrize("nd", [9, 5])
def test_msi_ieee_fallback_on_extreme_magnitudes(nd):
    """A fifth of the equations scaled by 2^-1015 (the exact solution does not
    change): the remainders of their factors' reciprocal-based (Markstein)
    quotients fall into the subnormal range, where such a quotient need not
    be the IEEE one.  Every factor is checked against IEEE division and the
    factorisation repeated with it, so the solve stays bitwise the oracle's,
    and the repetition is counted."""
    nx, ny = 47, 70
    a, b = random_dominant_planes(nd, nx, ny, seed=21)
    rows = np.random.default_rng(22).random(nx * ny) < 0.2
    scale = np.where(rows, 2.0 ** -1015, 1.0)
    a = (a.reshape(nd, -1) * scale).reshape(-1).copy()
    b = b * scale
    from mach2d_b200._lib import lib
    L = lib()
    L.m2d_msi_lu_redo_count.restype = ctypes.c_longlong
    before = L.m2d_msi_lu_redo_count()
    x0 = np.random.default_rng(23).standard_normal(nx * ny)
    xg, xo = x0.copy(), x0.copy()
    nit_g = _gpu_msi(nd, nx, ny, 4, 1e-30, a, b, xg)
    nit_o = orc(f"msi{nd}_solve", nx, ny, 4, 1e-30, a, b, xo)
    assert nit_g == nit_o
    assert np.array_equal(xg, xo), np.max(np.abs(xg - xo))
    assert L.m2d_msi_lu_redo_count() > before


@pytest.mark.parametrize("nd", [9, 5])
def test_msi_more_rows_than_threads(nd):
    # ny > 1024: each thread owns two rows of the wavefront
    nx, ny = 9, 1100
    a, b = dirichlet_system(nd, nx, ny, seed=9)
    xg, xo = np.zeros(nx * ny), np.zeros(nx * ny)
    assert _gpu_msi(nd, nx, ny, 3, 1e-30, a, b, xg) == orc(f"msi{nd}_solve", nx, ny, 3, 1e-30, a, b, xo)
    assert np.array_equal(xg, xo)


@pytest.mark.parametrize("nd", [9, 5])
def test_msi_dirichlet_system_converges(nd):
    nx, ny = 258, 130
    a, b = dirichlet_system(nd, nx, ny, seed=21)
    xg, xo = np.zeros(nx * ny), np.zeros(nx * ny)
    nit_g = _gpu_msi(nd, nx, ny, 200, 1e-10, a, b, xg)
    nit_o = orc(f"msi{nd}_solve", nx, ny, 200, 1e-10, a, b, xo)
    assert nit_g == nit_o and nit_g < 200
    assert np.array_equal(xg, xo)


@pytest.mark.parametrize("nd", [9, 5])
@pytest.mark.parametrize("nx,ny,nitm", [(8, 6, 1), (45, 23, 3), (200, 100, 5)])
def test_tdma_bitwise(nd, nx, ny, nitm):
    a, b = random_dominant_planes(nd, nx, ny, seed=nx)
    x0 = np.random.default_rng(nx).standard_normal(nx * ny)
    xg, xo = x0.copy(), x0.copy()
    (ClassSolverTDMA9d if nd == 9 else ClassSolverTDMA5d)().init(nx, ny, nitm).solve(a, b, xg)
    orc(f"tdma2d{nd}", nx, ny, nitm, a, b, xo)
    assert np.array_equal(xg, xo)


def test_tdma_lines_bitwise():
    aw, ap, ae, d = tdma_lines_system(n=1024, nlines=512, seed=4)
    x = tdma_lines(aw, ap, ae, d)
    for l in (0, 1, 255, 511):
        xo = np.zeros(1024)
        orc("tdma_line", 1024, aw[l].copy(), ap[l].copy(), ae[l].copy(), d[l].copy(), xo)
        assert np.array_equal(x[l], xo)


@pytest.mark.parametrize("n,nlines", [(1024, 512), (1000, 37), (7, 5), (2048, 3)])
def test_tdma_lines_device_both_methods(n, nlines):
    """m2d_tdma_lines_device: method 0 (the sequential recurrence) bitwise the
    oracle's line sweep; method 1 (parallel cyclic reduction) within 1e-12
    of it relative to max|x| (the isolated-system lines, aP = 1.05 (|aW| +
    |aE|), are strongly diagonally dominant)."""
    import ctypes

    import torch
    from mach2d_b200._lib import check, lib
    dev = torch.device("cuda:0")
    aw, ap, ae, d = tdma_lines_system(n=n, nlines=nlines, seed=n + nlines)
    xo = np.zeros((nlines, n))
    for l in range(nlines):
        orc("tdma_line", n, aw[l].copy(), ap[l].copy(), ae[l].copy(), d[l].copy(), xo[l])
    L = lib()
    L.m2d_tdma_lines_device.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int,
                                                                                                ctypes.c_void_p]
    t = [torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (aw, ap, ae, d)]
    work = torch.empty(2 * n * nlines, dtype=torch.float64, device=dev)
    for method in (0, 1):
        x = torch.zeros(nlines, n, dtype=torch.float64, device=dev)
        check(L.m2d_tdma_lines_device(n, nlines, *[v.data_ptr() for v in t], x.data_ptr(), work.data_ptr(), method,
                                      None))
        xg = x.cpu().numpy()
        if method == 0:
            assert np.array_equal(xg, xo)
        else:
            assert np.max(np.abs(xg - xo)) <= 1e-12 * np.max(np.abs(xo))


def test_norms_match_oracle():
    nx, ny = 60, 31
    a9, b = random_dominant_planes(9, nx, ny, seed=5)
    a5, _ = random_dominant_planes(5, nx, ny, seed=6)
    x = np.random.default_rng(7).standard_normal(nx * ny)
    assert norm_l1_9d(nx, ny, x, b, a9, 1.5) == pytest.approx(orc("norm_l1_9d", nx, ny, x, b, a9, 1.5), rel=1e-12)
    assert norm_l1_5d(nx, ny, x, b, a5, 0.0) == pytest.approx(orc("norm_l1_5d", nx, ny, x, b, a5, 0.0), rel=1e-12)
    assert norm_l1_9d_relative(nx, ny, x, b, a9, 0.25) == pytest.approx(
        orc("norm_l1_9d_relative", nx, ny, x, b, a9, 0.25), rel=1e-12)


def test_zero_pivot_is_reported_not_trapped():
    nx, ny = 12, 10
    a, b = dirichlet_system(9, nx, ny, seed=1)
    a = a.reshape(9, -1)
    a[4, 5 * nx + 5] = 0.0
    a[:, 5 * nx + 5] = 0.0            # an empty row: zero pivot
    x = np.zeros(nx * ny)
    with pytest.raises(M2DError) as e:
        _gpu_msi(9, nx, ny, 2, 1e-2, a.reshape(-1).copy(), b, x)
    assert e.value.code == 7


def test_unbounded_iteration_stops_at_cap():
    nx, ny = 8, 6
    a, b = dirichlet_system(5, nx, ny, seed=2)
    x = np.zeros(nx * ny)
    nit = ctypes.c_int(0)
    with pytest.raises(M2DError) as e:
        call("m2d_msi5_solve_it", nx, ny, 0, 0.0, a, b, x, nit)   # tol 0: never converges
    assert e.value.code == 4
    assert nit.value == 0 or nit.value == 10000
