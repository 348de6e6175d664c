"""The external-flow boundary plug-in (src/user/external_flow/mod_extflow.f90:
166-317) against the oracle's restatement, bitwise.

Each drop-in writes the boundary rows of the far field (north), the body
wall (south: slip for Euler, no-slip for Navier-Stokes, adiabatic or
prescribed temperature), the outflow (east) and the symmetry axis (west),
corners included, exactly as the reference's strip schemes
(mod_extflow_procedures.f90:344-701) and transfer
(src/boundary_conditions/mach2d_bc9d.f90:521-706, mach2d_bc5d.f90:133-297)
leave them; interior rows keep the caller's values.  Seeded random metrics
and velocities; odd and small grids included.
"""
import ctypes

import numpy as np
import pytest

from _oracle import call as orc
from mach2d_b200._lib import call

pytestmark = pytest.mark.gpu
SIZES = [(37, 23), (5, 5), (4, 6), (130, 66)]


def _fields(nx, ny, seed):
    r = np.random.default_rng(seed)
    N = nx * ny
    f = {k: r.uniform(0.5, 2.0, N) * r.choice([-1.0, 1.0], N) for k in ("xk", "yk", "betae", "betan", "u", "v")}
    f["alphae"] = r.uniform(0.5, 2.0, N)
    f["gamman"] = r.uniform(0.5, 2.0, N)
    return f


def _mat(nd, nx, ny, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(nd * nx * ny), r.standard_normal(nx * ny)


@pytest.mark.parametrize("nx,ny", SIZES)
@pytest.mark.parametrize("modvis", [0, 1])
def test_set_bcu_bcv_bitwise(nx, ny, modvis):
    f = _fields(nx, ny, nx + ny + modvis)
    a0, b0 = _mat(9, nx, ny, 1)
    ag, bg, ao, bo = a0.copy(), b0.copy(), a0.copy(), b0.copy()
    call("m2d_extflow_set_bcu", nx, ny, modvis, 341.5, f["xk"], f["yk"], f["alphae"], f["betae"], f["u"], f["v"],
         ag, bg)
    orc("extflow_set_bcu", nx, ny, modvis, 341.5, f["xk"], f["yk"], f["alphae"], f["betae"], f["u"], f["v"], ao, bo)
    assert np.array_equal(ag, ao) and np.array_equal(bg, bo)
    ag, bg, ao, bo = a0.copy(), b0.copy(), a0.copy(), b0.copy()
    call("m2d_extflow_set_bcv", nx, ny, modvis, f["xk"], f["yk"], f["u"], f["v"], ag, bg)
    orc("extflow_set_bcv", nx, ny, modvis, f["xk"], f["yk"], f["u"], f["v"], ao, bo)
    assert np.array_equal(ag, ao) and np.array_equal(bg, bo)
    # interior rows untouched
    A = ag.reshape(9, ny, nx)
    assert np.array_equal(A[:, 1:-1, 1:-1], a0.reshape(9, ny, nx)[:, 1:-1, 1:-1])


@pytest.mark.parametrize("nx,ny", SIZES)
@pytest.mark.parametrize("Tsbc", [-1.0, 300.0])
def test_set_bcT_and_bcpl_bitwise(nx, ny, Tsbc):
    f = _fields(nx, ny, 7 * nx + ny)
    a0, b0 = _mat(9, nx, ny, 2)
    ag, bg, ao, bo = a0.copy(), b0.copy(), a0.copy(), b0.copy()
    call("m2d_extflow_set_bcT", nx, ny, 288.15, Tsbc, f["alphae"], f["betae"], f["betan"], f["gamman"], ag, bg)
    orc("extflow_set_bcT", nx, ny, 288.15, Tsbc, f["alphae"], f["betae"], f["betan"], f["gamman"], ao, bo)
    assert np.array_equal(ag, ao) and np.array_equal(bg, bo)
    a0, b0 = _mat(5, nx, ny, 3)
    ag, bg, ao, bo = a0.copy(), b0.copy(), a0.copy(), b0.copy()
    call("m2d_extflow_set_bcpl", nx, ny, ag, bg)
    orc("extflow_set_bcpl", nx, ny, ao, bo)
    assert np.array_equal(ag, ao) and np.array_equal(bg, bo)


@pytest.mark.parametrize("nx,ny", SIZES)
def test_set_bcro_strips_bitwise(nx, ny):
    f = _fields(nx, ny, 3 * nx + ny)
    g = [np.zeros(9 * nx), np.zeros(9 * nx), np.zeros(9 * ny), np.zeros(9 * ny),
         np.zeros(nx), np.zeros(nx), np.zeros(ny), np.zeros(ny)]
    o = [v.copy() for v in g]
    call("m2d_extflow_set_bcro", nx, ny, 1.225, f["alphae"], f["betae"], f["betan"], f["gamman"], *g)
    orc("extflow_scheme_ro", nx, ny, 1.225, f["alphae"], f["betae"], f["betan"], f["gamman"], *o)
    for k, (x, y) in enumerate(zip(g, o)):
        assert np.array_equal(x, y), k


@pytest.mark.parametrize("nx,ny", SIZES + [(2050, 514)])
@pytest.mark.parametrize("modvis", [0, 1])
@pytest.mark.parametrize("itemax", [1, 3])
def test_extrapolate_u_v_bitwise(nx, ny, modvis, itemax):
    """extflow_extrapolate_u_v_to_fictitious (mod_extflow.f90:360-397): the
    ring cells of u, then of v, by itemax sweeps of boundary-line tridiagonal
    solves; interior cells untouched."""
    f = _fields(nx, ny, 11 * nx + ny + modvis)
    ug, vg, uo, vo = f["u"].copy(), f["v"].copy(), f["u"].copy(), f["v"].copy()
    call("m2d_extflow_extrapolate_u_v_to_fictitious", nx, ny, modvis, itemax, 341.5, f["xk"], f["yk"],
         f["alphae"], f["betae"], ug, vg)
    orc("extflow_extrapolate_u_v", nx, ny, modvis, itemax, 341.5, f["xk"], f["yk"], f["alphae"], f["betae"], uo, vo)
    assert np.array_equal(ug, uo) and np.array_equal(vg, vo)
    U = ug.reshape(ny, nx)
    assert np.array_equal(U[1:-1, 1:-1], f["u"].reshape(ny, nx)[1:-1, 1:-1])


@pytest.mark.parametrize("nx,ny", SIZES + [(2050, 514)])
@pytest.mark.parametrize("itemax", [0, 1, 4])
def test_extrapolate_ro_bitwise(nx, ny, itemax):
    """extflow_extrapolate_ro_to_fictitious (mod_extflow.f90:401-431)."""
    f = _fields(nx, ny, 13 * nx + ny)
    ro0 = np.random.default_rng(nx).uniform(0.5, 2.0, nx * ny)
    rg, ro = ro0.copy(), ro0.copy()
    call("m2d_extflow_extrapolate_ro_to_fictitious", nx, ny, itemax, 1.225, f["alphae"], f["betae"], f["betan"],
         f["gamman"], rg)
    orc("extflow_extrapolate_ro", nx, ny, itemax, 1.225, f["alphae"], f["betae"], f["betan"], f["gamman"], ro)
    assert np.array_equal(rg, ro)
    if itemax == 0:
        assert np.array_equal(rg, ro0)



@pytest.mark.parametrize("nx,ny", [(37, 23), (4, 6), (5000, 5)])
@pytest.mark.parametrize("modvis", [0, 1])
def test_calc_main_variables_bitwise(nx, ny, modvis):
    """extflow_calc_main_variables (mod_extflow.f90:321-356): the foredrag
    sums of get_cdfi / get_cdfv over i = 2..iocs, in the reference's order
    (the 5000-wide grid spans several summand chunks)."""
    f = _fields(nx, ny, 17 * nx + modvis)
    r = np.random.default_rng(nx + 1)
    N = nx * ny
    rn, Jn, vln = r.uniform(0.1, 1.0, N), r.uniform(0.5, 2.0, N), r.uniform(1e-5, 2e-5, N)
    p, Vcn = r.uniform(9e4, 1.1e5, N), r.standard_normal(N)
    for iocs in sorted({1, 2, nx // 2, nx}):
        cdfi, cdfv = ctypes.c_double(7.0), ctypes.c_double(7.0)
        call("m2d_extflow_calc_main_variables", nx, ny, 287.0, modvis, 1.0e5, 288.0, 340.0, 0.05, iocs,
             f["xk"], f["yk"], rn, Jn, vln, p, f["u"], f["v"], Vcn, cdfi, cdfv)
        cd = np.zeros(2)
        orc("extflow_calc_main_variables", nx, ny, 287.0, modvis, 1.0e5, 288.0, 340.0, 0.05, iocs,
            f["xk"], f["yk"], rn, Jn, vln, p, f["u"], f["v"], Vcn, cd)
        assert (cdfi.value, cdfv.value) == (cd[0], cd[1]), iocs
        if modvis == 0:
            assert cdfv.value == 0.0


@pytest.mark.parametrize("nx,ny", SIZES)
def test_boundary_T_from_H_bitwise(nx, ny):
    """extflow_boundary_T_from_H_conservation (mod_extflow.f90:438-544)."""
    r = np.random.default_rng(19 * nx + ny)
    N = nx * ny
    u, ue, un, v, ve, vn = (r.uniform(-300.0, 300.0, N) for _ in range(6))
    tg, to = np.zeros(N), np.zeros(N)
    bg = [np.full(ny, -1.0), np.full(ny, -1.0), np.full(nx, -1.0), np.full(nx, -1.0)]
    bo = [b.copy() for b in bg]
    call("m2d_extflow_boundary_T_from_H_conservation", nx, ny, 1004.5, 3.4e5, u, ue, un, v, ve, vn, tg, *bg)
    orc("extflow_boundary_T_from_H", nx, ny, 1004.5, 3.4e5, u, ue, un, v, ve, vn, to, *bo)
    assert np.array_equal(tg, to)
    for x, y in zip(bg, bo):
        assert np.array_equal(x, y) and x[0] == -1.0 and x[-1] == -1.0
