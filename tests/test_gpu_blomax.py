"""Baldwin-Lomax eddy viscosity (src/equations/blomax.f90) against the oracle.

The GPU kernel evaluates every per-cell expression with the reference's
operand order and replaces the per-line loops by warp reductions whose results
do not depend on order (max, first index of the maximum, first sign change),
so it matches the oracle to the last bits except where the device exp()
differs from the host's; the tolerance is 1e-12 relative.  The line-wide
decisions (location of F_max, inner/outer switch) must agree exactly, which
the fixtures make unambiguous.
"""
import numpy as np
import pytest

from _oracle import call as orc
from mach2d_b200._lib import call
from mach2d_b200.simplec import Simplec, euler_cosine_case

pytestmark = pytest.mark.gpu


def _grid_and_flow(nxr, nyr, seed):
    g = Simplec(euler_cosine_case(nxr, nyr))
    f = {k: g.field(k).copy() for k in ("x", "y", "xp", "yp", "xk", "yk", "Jp", "Jn")}
    nx, ny = g.nx, g.ny
    g.close()
    rng = np.random.default_rng(seed)
    yp = f["yp"].reshape(ny, nx)
    ywall = yp[ny - 2:ny - 1, :]                         # last real row, next to the north wall
    d = np.maximum(ywall - yp, 0.0) + 1e-4
    delta = 0.02 * (1.0 + 0.5 * np.linspace(0, 1, nx))[None, :]
    u = 300.0 * np.tanh(d / delta) * (1.0 + 0.05 * rng.standard_normal((ny, nx)))
    v = 5.0 * np.sin(3.0 * f["xp"].reshape(ny, nx)) * (1.0 + 0.05 * rng.standard_normal((ny, nx)))
    ro = 1.2 + 0.1 * rng.random((ny, nx))
    f.update(u=u.reshape(-1).copy(), v=v.reshape(-1).copy(), ro=ro.reshape(-1).copy(),
             ron=(ro * 1.01).reshape(-1).copy(),
             vln=(1.8e-5 * (1.0 + 0.01 * rng.random((ny, nx)))).reshape(-1).copy())
    return nx, ny, f


def _both(nx, ny, f):
    args = [f[k] for k in ("x", "y", "xp", "yp", "xk", "yk", "Jp", "Jn", "vln", "ro", "ron", "u", "v")]
    vg = np.full(nx * ny, -7.0)
    vo = vg.copy()
    call("m2d_get_eddy_viscosity_blomax", nx, ny, *args, vg)
    orc("get_eddy_viscosity_blomax", nx, ny, *args, vo, np.zeros(9 * (ny - 2)))
    return vg, vo


@pytest.mark.parametrize("nxr,nyr,seed", [(40, 20, 1), (128, 64, 2), (512, 256, 3)])
def test_blomax_matches_oracle(nxr, nyr, seed):
    nx, ny, f = _grid_and_flow(nxr, nyr, seed)
    vg, vo = _both(nx, ny, f)
    real = np.zeros((ny, nx), bool)
    real[1:-1, 1:-1] = True
    real = real.reshape(-1)
    assert np.all(vg[~real] == -7.0)                    # ghosts untouched, as intent(out) on reals only
    assert np.all(np.isfinite(vo[real])) and np.max(vo[real]) > 0
    scale = np.max(np.abs(vo[real]))
    assert np.max(np.abs(vg[real] - vo[real])) <= 1e-12 * scale


def test_blomax_zero_vorticity_gives_zero():
    nx, ny, f = _grid_and_flow(40, 20, 4)
    f["u"][:] = 100.0                                    # uniform flow: no vorticity, non-zero wall shear
    f["v"][:] = 0.0
    vg, vo = _both(nx, ny, f)
    assert np.array_equal(vg, vo)
    real = np.zeros((ny, nx), bool)
    real[1:-1, 1:-1] = True
    assert np.all(vg.reshape(ny, nx)[real] == 0.0)


def test_blomax_coefficients_round_trip_and_take_effect():
    nx, ny, f = _grid_and_flow(40, 20, 5)
    vg0, _ = _both(nx, ny, f)
    call("m2d_set_blomax_coefficients", 0.41, 26.0, 0.0168, 1.6, 0.3, 1.0)
    orc("set_blomax_coefficients", 0.41, 26.0, 0.0168, 1.6, 0.3, 1.0)
    try:
        vg1, vo1 = _both(nx, ny, f)
        import ctypes
        got = [ctypes.c_double() for _ in range(6)]
        call("m2d_get_blomax_coefficients", *got)
        assert [g.value for g in got] == [0.41, 26.0, 0.0168, 1.6, 0.3, 1.0]
        assert not np.array_equal(vg0, vg1)
        real = np.zeros((ny, nx), bool)
        real[1:-1, 1:-1] = True
        real = real.reshape(-1)
        assert np.max(np.abs(vg1[real] - vo1[real])) <= 1e-12 * np.max(np.abs(vo1[real]))
    finally:
        call("m2d_set_blomax_coefficients", 0.40, 26.0, 0.0168, 1.6, 0.3, 1.0)
        orc("set_blomax_coefficients", 0.40, 26.0, 0.0168, 1.6, 0.3, 1.0)


def test_eddy_viscosity_fictitious_bitwise():
    nx, ny = 37, 19
    phi = np.random.default_rng(6).standard_normal(nx * ny)
    pg, po = phi.copy(), phi.copy()
    call("m2d_get_eddy_viscosity_fictitious", nx, ny, pg)
    orc("get_eddy_viscosity_fictitious", nx, ny, po)
    assert np.array_equal(pg, po)
