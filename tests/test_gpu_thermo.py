"""Gas-mixture thermophysical model (src/thermophysical/) against the oracle.

cp, gamma and the boundary averages are polynomial or plain arithmetic in the
reference's operand order: bitwise.  Viscosity and conductivity go through
exp() and log(), whose device and host versions may differ in the last bit,
so they are compared to 1e-12 relative; the harmonic face means inside the
domain take the node values as input and are bitwise.

The species coefficients are synthetic (shaped like NASA-polynomial and
transport fits of diatomic and triatomic gases), seeded, so nothing here reads
a data file.
"""
import ctypes

import numpy as np
import pytest

from _oracle import call as orc
from mach2d_b200._lib import M2DError, call, lib
from mach2d_b200.thermo import Mixture, mixture_eval, mixture_init


def synthetic_species(n, seed):
    rng = np.random.default_rng(seed)
    Mi = rng.uniform(0.004, 0.044, n)
    # cp/R = a0 + a1 T (1 - c2 T + c3 T^2 - c4 T^3): positive on each range
    a1 = rng.uniform(0.0, 9e-3, n)
    cpl = np.column_stack([rng.uniform(2.5, 3.8, n), a1, -a1 * rng.uniform(0.6, 0.8, n) * 1e-3,
                           a1 * rng.uniform(0.2, 0.3, n) * 1e-6, -a1 * rng.uniform(0.0, 0.02, n) * 1e-9])
    a1 = rng.uniform(1e-4, 3e-3, n)
    cpu = np.column_stack([rng.uniform(2.9, 4.7, n), a1, -a1 * rng.uniform(0.3, 0.4, n) * 1e-3,
                           a1 * rng.uniform(0.05, 0.06, n) * 1e-6, -a1 * rng.uniform(0.003, 0.004, n) * 1e-9])
    vl = np.column_stack([rng.uniform(0.54, 0.83, n), rng.uniform(-190, 120, n), rng.uniform(-1e4, 9e3, n),
                          rng.uniform(0.7, 2.5, n)])
    vu = np.column_stack([rng.uniform(0.62, 0.66, n), rng.uniform(-150, 55, n), rng.uniform(-8e4, -1.6e4, n),
                          rng.uniform(1.5, 2.2, n)])
    kl, ku = vl * rng.uniform(0.9, 1.1, (n, 4)), vu * rng.uniform(0.9, 1.1, (n, 4))
    return Mi, np.hstack([cpl, cpu]), np.hstack([vl, vu]), np.hstack([kl, ku])


def both_mixtures(base, fr, seed):
    Mi, cpi, mui, kpi = synthetic_species(len(fr), seed)
    fr = np.asarray(fr, dtype=np.float64)
    mg = mixture_init(base, fr, Mi, cpi, mui, kpi)
    mo = Mixture()
    rc = orc("mixture_init", base, len(fr), fr, Mi.copy(), cpi.reshape(-1).copy(), mui.reshape(-1).copy(),
             kpi.reshape(-1).copy(), ctypes.byref(mo))
    assert rc == 0
    return mg, mo


MIXES = [(0, [0.79, 0.21], 1), (1, [0.7, 0.2, 0.1], 2), (0, [0.5, 1e-9, 0.25, 0.25], 3),
         (1, [0.125] * 8, 4), (0, [1.0], 5)]


def _orc_scalar(name, m, T):
    f = getattr(__import__("_oracle").lib(), "orc_mix_" + name)
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.POINTER(Mixture), ctypes.c_double]
    return f(ctypes.byref(m), T)


@pytest.mark.parametrize("base,fr,seed", MIXES)
def test_mixture_init_and_point_values_match_oracle(base, fr, seed):
    """Host side of the library (no GPU): init and point values."""
    mg, mo = both_mixtures(base, fr, seed)
    assert bytes(mg) == bytes(mo)                       # same layout, same bits
    assert mg.ngs == sum(1 for f in fr if f > 1e-8)
    for T in (200.0, 300.0, 999.0, 1000.0, 1000.5, 2500.0):
        cp, mu, kp, gm = mixture_eval(mg, T)
        assert cp == _orc_scalar("cp", mo, T) and gm == _orc_scalar("gm", mo, T)
        assert mu == _orc_scalar("mu", mo, T) and kp == _orc_scalar("kp", mo, T)
        assert cp > mg.Rg > 0 and mu > 0 and kp > 0


def test_mixture_init_rejects_bad_fractions():
    Mi, cpi, mui, kpi = synthetic_species(2, 9)
    with pytest.raises(M2DError) as e:
        mixture_init(0, [0.5, 0.4], Mi, cpi, mui, kpi)
    assert e.value.code == 2
    with pytest.raises(M2DError):
        mixture_init(1, [0.0, 0.0], Mi, cpi, mui, kpi)


def _fields(nx, ny, seed):
    rng = np.random.default_rng(seed)
    T = rng.uniform(250.0, 2500.0, nx * ny)
    Tb = [0.5 * (rng.uniform(250.0, 2500.0, n) + 900.0) for n in (nx, nx, ny, ny)]
    return T, Tb


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny", [(7, 5), (66, 34), (514, 130)])
def test_boundary_fields_bitwise(nx, ny):
    F = np.random.default_rng(nx).standard_normal(nx * ny)
    g = [np.full(n, -3.0) for n in (nx, nx, ny, ny)]
    o = [a.copy() for a in g]
    call("m2d_get_boundary_fields", nx, ny, F, *g)
    orc("get_boundary_fields", nx, ny, F, *o)
    for a, b in zip(g, o):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("base,fr,seed", MIXES[:4])
@pytest.mark.parametrize("nx,ny", [(6, 5), (130, 66)])
def test_set_cp_and_gamma_bitwise(base, fr, seed, nx, ny):
    mg, mo = both_mixtures(base, fr, seed)
    T, (Tbn, Tbs, Tbe, Tbw) = _fields(nx, ny, seed)
    cg = np.full(nx * ny, -1.0)
    co = cg.copy()
    call("m2d_set_cp", mg, nx, ny, Tbn, Tbs, Tbe, Tbw, T, cg)
    orc("set_cp", ctypes.byref(mo), nx, ny, Tbn, Tbs, Tbe, Tbw, T, co)
    assert np.array_equal(cg, co)
    assert np.all(co > 0)
    gg, go = np.zeros(nx * ny), np.zeros(nx * ny)
    call("m2d_set_gamma", nx, ny, float(mg.Rg), cg, gg)
    orc("set_gamma", nx, ny, float(mo.Rg), co, go)
    assert np.array_equal(gg, go)
    assert np.all((go > 1.0) & (go < 1.7))


def _close(a, b, tol=1e-12):
    return np.max(np.abs(a - b) / np.abs(b)) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("visc", [True, False])
@pytest.mark.parametrize("base,fr,seed", MIXES)
def test_transport_nodes_and_faces(visc, base, fr, seed):
    nx, ny = 98, 35
    mg, mo = both_mixtures(base, fr, seed)
    T, Tb = _fields(nx, ny, seed + 10)
    node = "m2d_set_laminar_viscosity_at_nodes" if visc else "m2d_set_thermal_conductivity_at_nodes"
    face = "m2d_get_laminar_viscosity_at_faces" if visc else "m2d_get_thermal_conductivity_at_faces"
    pg = np.full(nx * ny, 7.0)
    po = pg.copy()
    call(node, mg, nx, ny, T, pg)
    orc("transport_nodes", ctypes.byref(mo), nx, ny, int(visc), T, po)
    real = np.zeros((ny, nx), bool)
    real[1:-1, 1:-1] = True
    real = real.reshape(-1)
    assert np.all(pg[~real] == 7.0)
    assert _close(pg[real], po[real])
    # faces from the same node values: interior harmonic means bitwise
    eg, ng = np.full(nx * ny, -1.0), np.full(nx * ny, -1.0)
    eo, no = eg.copy(), ng.copy()
    call(face, mg, nx, ny, *Tb, po, eg, ng)
    orc("transport_faces", ctypes.byref(mo), nx, ny, int(visc), *Tb, po, eo, no)
    e2, n2 = eg.reshape(ny, nx), ng.reshape(ny, nx)
    e2o, n2o = eo.reshape(ny, nx), no.reshape(ny, nx)
    assert np.array_equal(e2[1:-1, 1:-2], e2o[1:-1, 1:-2])
    assert np.array_equal(n2[1:-2, 1:-1], n2o[1:-2, 1:-1])
    assert _close(e2[1:-1, [0, nx - 2]], e2o[1:-1, [0, nx - 2]])
    assert _close(n2[[0, ny - 2], 1:-1], n2o[[0, ny - 2], 1:-1])
    touched = np.zeros((ny, nx), bool)
    touched[1:-1, 0:nx - 1] = True
    assert np.all(e2[~touched] == -1.0)
    touched = np.zeros((ny, nx), bool)
    touched[0:ny - 1, 1:-1] = True
    assert np.all(n2[~touched] == -1.0)


def test_library_exports_thermo_entry_points():
    for s in ("m2d_mixture_init", "m2d_mixture_eval", "m2d_set_cp", "m2d_set_gamma",
              "m2d_set_laminar_viscosity_at_nodes", "m2d_set_thermal_conductivity_at_nodes",
              "m2d_get_laminar_viscosity_at_faces", "m2d_get_thermal_conductivity_at_faces",
              "m2d_get_boundary_fields"):
        assert hasattr(lib(), s)
