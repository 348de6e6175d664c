"""Flexible GMRES around the MSI factorisation (m2d_fgmres_solve), no
counterpart in the reference (which iterates MSI as a stationary method,
src/solvers/msi2d9-v03.f90:42-262).

The solver's own residual estimate is checked against the true residual of
the returned x, recomputed here in numpy from the coefficient planes: it
must meet the requested relative tolerance.  On the isolated-system
workload (off-diagonals U[-1, 0], aP = 1.05 sum|a_nb|, zero-Dirichlet ring)
the Krylov iteration needs fewer MSI sweep pairs than MSI iterated alone
to the same tolerance -- which also shows that the factors each step reuses
are the right ones (stale or wrong factors would cost many more steps).
"""
import numpy as np
import pytest

from _systems import dirichlet_system, offsets
from mach2d_b200._lib import M2DError
from mach2d_b200.solvers import fgmres

pytestmark = pytest.mark.gpu


def _residual(nd, nx, ny, a, b, x):
    A = a.reshape(nd, ny, nx)
    X = x.reshape(ny, nx)
    r = b.reshape(ny, nx).copy()
    for k, (di, dj) in enumerate(offsets(nd)):
        sh = np.zeros_like(X)
        ys, ye = max(0, -dj), ny - max(0, dj)
        xs, xe = max(0, -di), nx - max(0, di)
        sh[ys:ye, xs:xe] = X[ys + dj:ye + dj, xs + di:xe + di]
        r -= A[k] * sh
    return np.linalg.norm(r) / np.linalg.norm(b)


def _plain_msi_iterations(nd, nx, ny, a, b, tol):
    import ctypes
    from mach2d_b200._lib import call
    x = np.zeros(nx * ny)
    nit = ctypes.c_int()
    call(f"m2d_msi{nd}_solve_it", nx, ny, 5000, tol, a, b, x, nit)
    return nit.value


@pytest.mark.parametrize("nd", [9, 5])
@pytest.mark.parametrize("prec", [0, 1])
def test_fgmres_meets_tolerance_with_fewer_msi_sweeps(nd, prec):
    import torch
    dev = torch.device("cuda:0")
    nx, ny, tol = 194, 98, 1e-10
    a, b = dirichlet_system(nd, nx, ny, seed=61 + nd)
    da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    rep = fgmres(nd, nx, ny, da, db, x, tol, prec=prec, restart=30)
    assert rep.converged == 1 and rep.rel_residual <= tol * 1.0001
    assert _residual(nd, nx, ny, a, b, x.cpu().numpy()) <= tol * 1.001
    plain = _plain_msi_iterations(nd, nx, ny, a, b, tol)
    assert rep.msi_applications == rep.iterations
    assert rep.msi_applications < plain, (rep.msi_applications, plain)


def test_fgmres_is_reproducible_and_reports_the_iteration_cap():
    import torch
    dev = torch.device("cuda:0")
    nx, ny = 98, 66
    a, b = dirichlet_system(9, nx, ny, seed=70)
    da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    xs = []
    for _ in range(2):
        x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
        fgmres(9, nx, ny, da, db, x, 1e-11, prec=0, restart=8)
        xs.append(x.cpu().numpy())
    assert np.array_equal(xs[0], xs[1])
    x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    with pytest.raises(M2DError) as e:
        fgmres(9, nx, ny, da, db, x, 1e-14, prec=0, restart=4, maxit=3)
    assert e.value.code == 4


def test_learned_preconditioner_cuts_msi_applications():
    """The learned correction as FGMRES's preconditioner (prec 2: z = N(v),
    then one FP32 MSI step from it), the network trained here by the
    library's kernels on the MSI solutions of 16 other seeds of the same
    5-diagonal isolated system: it meets the tolerance with fewer MSI sweep
    pairs than MSI iterated alone and than FGMRES with MSI alone."""
    import torch
    from _systems import isolated5
    from mach2d_b200 import unet
    dev = torch.device("cuda:0")
    nx, ny, tol = 258, 130, 1e-10
    H, W = unet.image_shape(nx, ny)
    Jp = torch.ones(nx * ny, dtype=torch.float64, device=dev)
    systems = [tuple(torch.from_numpy(v).to(dev) for v in isolated5(nx, ny, seed=200 + s)) for s in range(16)]
    pairs = unet.PairSet(16, H, W)
    unet.harvest_systems(systems, nx, ny, Jp, pairs)
    net = unet.UNet(8, H, W, seed=1)
    hist = unet.train(net, pairs, 400, batch=8, lr=2e-3, lr_final=1e-4)
    assert np.mean(hist[-20:]) < 0.5 * hist[0]
    one = unet.UNet(1, H, W, params=net.params())
    net.close()
    a, b = isolated5(nx, ny, seed=7)
    da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    r2 = fgmres(5, nx, ny, da, db, x, tol, prec=2, net=one, Jp=Jp)
    assert r2.converged == 1 and r2.learned_applications == r2.iterations
    assert _residual(5, nx, ny, a, b, x.cpu().numpy()) <= tol * 1.001
    x1 = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    r1 = fgmres(5, nx, ny, da, db, x1, tol, prec=1)
    plain = _plain_msi_iterations(5, nx, ny, a, b, tol)
    assert r2.msi_applications < r1.msi_applications < plain, (r2.msi_applications, r1.msi_applications, plain)
    one.close()
