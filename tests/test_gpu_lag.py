"""Lagged factorisation (m2d_case.msi_lag) and the device solve's explicit
options (m2d_msi_solve_device_ex).

* The FP64 solve with reused factors gives the fresh solve's iterates,
  bitwise: reuse skips only the transpose of A and the factorisation, and
  the initial residual (computed then by every warp instead of the helper
  warps) has the same per-thread sums and tree.
* msi_lag leaves the FP64 solver (0) bitwise unchanged: lagging applies to
  FP32 factors only.
* With FP32 sweeps and msi_lag = 16 the outer iterations are deterministic
  (two runs bitwise equal) and stay on the unlagged run's track: each solve
  passes the same FP64 stopping test with an older preconditioner.
"""
import ctypes

import numpy as np
import pytest
import torch

from _systems import isolated5
from mach2d_b200._lib import check, lib
from mach2d_b200.simplec import Simplec, euler_cosine_case

pytestmark = pytest.mark.gpu


def _ex(nd, nx, ny, a, b, x, work, nit, prec, reuse, nitm=50, tol=1e-10):
    L = lib()
    L.m2d_msi_solve_device_ex.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
                                          + [ctypes.c_int] * 2 + [ctypes.c_void_p])
    check(L.m2d_msi_solve_device_ex(nd, nx, ny, nitm, tol, a.data_ptr(), b.data_ptr(), x.data_ptr(),
                                    work.data_ptr(), torch.cuda.current_stream().cuda_stream, nit.data_ptr(),
                                    prec, reuse, None))
    torch.cuda.synchronize()


@pytest.mark.parametrize("prec", [0, 1])
def test_reused_factors_give_the_fresh_iterates(prec):
    nx, ny = 130, 66
    a, b = isolated5(nx, ny, seed=3)
    a, b = torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda")
    L = lib()
    L.m2d_msi_workspace_doubles.restype = ctypes.c_long
    work = torch.zeros(L.m2d_msi_workspace_doubles(5, nx, ny), dtype=torch.float64, device="cuda")
    nit = torch.zeros(1, dtype=torch.int32, device="cuda")
    x1 = torch.zeros(nx * ny, dtype=torch.float64, device="cuda")
    _ex(5, nx, ny, a, b, x1, work, nit, prec, 0)
    n1 = int(nit.item())
    x2 = torch.zeros_like(x1)
    _ex(5, nx, ny, a, b, x2, work, nit, prec, 1)
    assert int(nit.item()) == n1 > 1
    assert torch.equal(x1, x2)


def test_ex_rejects_bad_options():
    L = lib()
    L.m2d_msi_solve_device_ex.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
                                          + [ctypes.c_int] * 2 + [ctypes.c_void_p])
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert L.m2d_msi_solve_device_ex(5, 8, 8, 1, 1e-2, p, p, p, p, None, None, 2, 0, None) == 2
    assert L.m2d_msi_solve_device_ex(5, 8, 8, 1, 1e-2, p, p, p, p, None, None, 0, 3, None) == 2


def _run(solver, lag, iters=300, **over):
    c = euler_cosine_case(64, 32, solver=solver, **over)
    c.msi_lag = lag
    g = Simplec(c)
    g.set_graph(True)
    reps = [g.iterate() for _ in range(iters)]
    out = {f: g.field(f) for f in ("u", "v", "p", "T")}
    g.close()
    return reps, out


def test_lag_leaves_fp64_unchanged():
    r0, f0 = _run(0, 0, 60)
    r1, f1 = _run(0, 16, 60)
    assert [r.normpl for r in r0] == [r.normpl for r in r1]
    for k in f0:
        assert np.array_equal(f0[k], f1[k]), k


def test_lagged_fp32_is_deterministic_and_on_track():
    ra, fa = _run(2, 16)
    rb, fb = _run(2, 16)
    assert [r.normpl for r in ra] == [r.normpl for r in rb]
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k
    r2, f2 = _run(2, 0)
    assert ra[-1].it == r2[-1].it
    ratios = [x.normpl / y.normpl for x, y in zip(ra, r2)]
    assert 0.5 < float(np.exp(np.mean(np.log(ratios)))) < 2.0
    for k in fa:
        assert np.max(np.abs(fa[k] - f2[k])) <= 1e-2 * np.max(np.abs(f2[k])), k


def test_lagged_fp32_navier_stokes_keeps_each_equations_factors():
    """Navier-Stokes: u, v, T and p' each keep their own factor record and
    workspace, so the energy equation's solve neither reuses nor overwrites
    the u factors; the run stays deterministic and on the unlagged run's
    track."""
    ns = dict(modvis=1, Twall=900.0)
    ra, fa = _run(2, 16, 200, **ns)
    rb, fb = _run(2, 16, 200, **ns)
    assert [r.normpl for r in ra] == [r.normpl for r in rb]
    r2, f2 = _run(2, 0, 200, **ns)
    ratios = [x.normpl / y.normpl for x, y in zip(ra, r2)]
    assert 0.5 < float(np.exp(np.mean(np.log(ratios)))) < 2.0
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k
        assert np.max(np.abs(fa[k] - f2[k])) <= 1e-2 * np.max(np.abs(f2[k])), k
