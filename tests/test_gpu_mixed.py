"""MSI with FP32 factors and sweeps inside the FP64 iteration ("MSI_MIXED").

No counterpart in the reference and not bitwise: the contract is that the
FP64 iteration still converges to the FP64 solution.  The residual
r = b - A x of the returned x is re-evaluated here in FP64 (numpy) and must
meet the requested relative tolerance; the iteration count stays close to
the FP64 solve's (the FP32 incomplete LU preconditions as well as the FP64
one to about single precision); and a whole nozzle run with the mixed solver
converges to the same integrals as the FP64 reference path.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from _systems import dirichlet_system, offsets
from mach2d_b200._lib import call
from mach2d_b200.simplec import Simplec, n01_case
from mach2d_b200.solvers import solvers_init

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.json")


def apply(a, x, nd, nx, ny):
    """A x for plane-major coefficients (neighbours outside the grid skipped)."""
    a = a.reshape(nd, ny, nx)
    X = x.reshape(ny, nx)
    y = np.zeros((ny, nx))
    for k, (di, dj) in enumerate(offsets(nd)):
        i0, i1 = max(0, -di), nx - max(0, di)
        j0, j1 = max(0, -dj), ny - max(0, dj)
        y[j0:j1, i0:i1] += a[k, j0:j1, i0:i1] * X[j0 + dj:j1 + dj, i0 + di:i1 + di]
    return y.reshape(-1)


def fast_dirichlet_system(nd, nx, ny, seed=0, dominance=1.05):
    """Vectorised form of _systems.dirichlet_system (same rule, other stream)."""
    rng = np.random.default_rng(seed)
    off = offsets(nd)
    kp = off.index((0, 0))
    a = np.zeros((nd, ny, nx))
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    interior = (ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < ny - 1)
    for k, (di, dj) in enumerate(off):
        if k == kp:
            continue
        ni, nj = ii + di, jj + dj
        ok = interior & (ni > 0) & (ni < nx - 1) & (nj > 0) & (nj < ny - 1)
        a[k] = np.where(ok, -rng.uniform(0.0, 1.0, (ny, nx)), 0.0)
    s = np.abs(a).sum(axis=0)
    a[kp] = np.where(interior & (s > 0), dominance * s, 1.0)
    b = np.where(interior, rng.standard_normal((ny, nx)), 0.0)
    return a.reshape(-1).copy(), b.reshape(-1).copy()


def _solve(name, nd, nx, ny, nitm, tol, a, b, x):
    nit = ctypes.c_int(0)
    call(name, nx, ny, nitm, tol, a, b, x, nit)
    return nit.value


@pytest.mark.parametrize("nd", [9, 5])
@pytest.mark.parametrize("nx,ny,gen", [(258, 130, "loop"), (1026, 514, "vec")])
def test_mixed_reaches_fp64_tolerance(nd, nx, ny, gen):
    # 1026 x 514 is the isolated-system size with its ghost ring (two
    # wavefront warps per CTA); 258 x 130 runs one warp per CTA
    a, b = (dirichlet_system if gen == "loop" else fast_dirichlet_system)(nd, nx, ny, seed=40 + nd)
    tol = 1e-10
    x64, xmx = np.zeros(nx * ny), np.zeros(nx * ny)
    n64 = _solve(f"m2d_msi{nd}_solve_it", nd, nx, ny, 5000, tol, a, b, x64)
    nmx = _solve(f"m2d_msi{nd}_solve_mixed", nd, nx, ny, 5000, tol, a, b, xmx)
    r0 = np.linalg.norm(b)
    assert np.linalg.norm(b - apply(a, x64, nd, nx, ny)) < tol * r0
    assert np.linalg.norm(b - apply(a, xmx, nd, nx, ny)) < tol * r0
    assert nmx <= n64 + max(2, n64 // 20), (nmx, n64)
    assert np.max(np.abs(xmx - x64)) <= 1e-8 * np.max(np.abs(x64))


def test_mixed_solver_factory_option():
    s5, s9 = solvers_init(66, 34, "MSI_MIXED", 5, 20, 1e-2, 1e-2)
    assert type(s9).__name__ == "ClassSolverMSIMixed9d" and type(s5).__name__ == "ClassSolverMSIMixed5d"
    a, b = dirichlet_system(9, 66, 34, seed=3)
    x = np.zeros(66 * 34)
    s9.solve(a, b, x)
    assert s9.nit >= 1 and np.all(np.isfinite(x))


def test_reference_deck_with_mixed_solver_reaches_golden_integrals():
    gold = json.load(open(GOLD))["n01_euler_20x10"]["final"]
    g = Simplec(n01_case(solver=2))
    rep = g.run(3000)
    assert rep.normpl < 1e-10
    fmi, fme, Fd, Cd, pwall = g.integrals()
    rel = lambda u, v: abs(u - v) / abs(v)
    assert rel(Cd, gold["Cd"]) < 1e-6
    assert rel(fme, gold["fme"]) < 1e-6 and rel(Fd, gold["Fd"]) < 1e-6
    assert np.max(np.abs(pwall - np.array(gold["pwall"])) / np.max(np.abs(gold["pwall"]))) < 1e-6
