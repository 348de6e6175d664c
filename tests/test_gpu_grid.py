"""Grid metrics (src/grid/mod_grid.f90:237-723) and the instance set-up on the
device against the oracle.

The drop-ins m2d_get_real_centroids_xy, m2d_get_metrics and m2d_get_radius
are plain FP64 arithmetic in the reference's order: bitwise, on the nozzle
grids of both contours and both node distributions and on randomly
perturbed grids, with every output element written (the outputs start as
NaN).  The set-up of a context (m2d_create) computes the metrics and every
O(nx ny) part of the initial guess on the device from the host's grid nodes
and quasi-1D strips: the whole initial state (every plane, strip and
reference scalar) is bitwise the oracle's, except the MIXTURE model's
viscosity and conductivity, which go through the device's exp and log
(1e-12 relative).
"""
import ctypes
import json
import os

import numpy as np
import pytest

from _oracle import OracleCase
from _oracle import call as orc
from _states import NAMES
from mach2d_b200._lib import call, lib
from mach2d_b200.simplec import Simplec, euler_cosine_case, n01_case

METRICS = ("xe", "ye", "xen", "yen", "xk", "yk", "xke", "yke", "Jp", "Je", "Jn",
           "alphae", "gamman", "betae", "betan")


def _air():
    from mach2d_b200.thermo import mixture_init
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "air_species.json")))
    return mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])


GRIDS = {
    "c01": lambda: euler_cosine_case(40, 20),
    "n01": lambda: n01_case(),
    "n01_pg": lambda: n01_case(36, 18, kg=2, a1=2e-4),
    "c01_pg_wide": lambda: euler_cosine_case(130, 33, kg=2, a1=1e-3),
}


def _grid(name, perturb=None):
    o = OracleCase(GRIDS[name]())
    x, y = o.field("x"), o.field("y")
    if perturb is not None:
        rng = np.random.default_rng(perturb)
        h = np.min(np.abs(np.diff(x.reshape(o.ny, o.nx)[1:-1, :-1], axis=1)))
        x = x + rng.uniform(-0.2, 0.2, x.size) * h
        y = y + rng.uniform(-0.2, 0.2, y.size) * h
    return o.nx, o.ny, x, y


def _nan(n, k):
    return [np.full(n, np.nan) for _ in range(k)]


@pytest.mark.gpu
@pytest.mark.parametrize("perturb", [None, 7])
@pytest.mark.parametrize("name", sorted(GRIDS))
def test_centroids_metrics_radius_bitwise(name, perturb):
    nx, ny, x, y = _grid(name, perturb)
    N = nx * ny
    for opt in (1, 2):
        g, o = _nan(N, 2), _nan(N, 2)
        call("m2d_get_real_centroids_xy", opt, nx, ny, x, y, *g)
        orc("get_real_centroids_xy", opt, nx, ny, x, y, *o)
        for a, b in zip(g, o):
            assert np.array_equal(a, b), opt
        xp, yp = o
        g, o = _nan(N, 15), _nan(N, 15)
        call("m2d_get_metrics", nx, ny, x, y, xp, yp, *g)
        orc("get_metrics", nx, ny, x, y, xp, yp, *o)
        for k, (a, b) in enumerate(zip(g, o)):
            assert np.array_equal(a, b), (opt, METRICS[k])
        for coord in (0, 1):
            g, o = _nan(N, 4), _nan(N, 4)
            call("m2d_get_radius", coord, nx, ny, y, yp, *g)
            orc("get_radius", coord, nx, ny, y, yp, *o)
            for k, (a, b) in enumerate(zip(g, o)):
                assert np.array_equal(a, b), (opt, coord, ("radius", "re", "rn", "rp")[k])


def test_grid_drop_ins_reject_small_grids_without_device_work():
    L = lib()
    n3, n9, one = ctypes.c_int(3), ctypes.c_int(9), ctypes.c_int(1)
    buf = (ctypes.c_double * 27)()
    assert L.m2d_get_real_centroids_xy(ctypes.byref(one), ctypes.byref(n3), ctypes.byref(n9),
                                       buf, buf, buf, buf) == 2
    assert L.m2d_get_radius(ctypes.byref(one), ctypes.byref(n9), ctypes.byref(n3), buf, buf,
                            buf, buf, buf, buf) == 2
    assert L.m2d_get_metrics(ctypes.byref(n3), ctypes.byref(n9), *([buf] * 21)) == 2


STATE_CASES = {
    "c01_euler": lambda: euler_cosine_case(40, 20),
    "n01_deck": lambda: n01_case(),
    "n01_pg_kcm2": lambda: n01_case(30, 14, kg=2, kcm=2, a1=2e-4),
    "c01_navier_stokes": lambda: euler_cosine_case(30, 14, modvis=1, Twall=900.0),
    "c01_planar": lambda: euler_cosine_case(24, 12, coord=0),
    "n01_ramp_dt": lambda: n01_case(dtmodel=0, dt1=1e-7, dt2=1e-6, it1=3, it2=10),
    "c01_mixture_ns": lambda: euler_cosine_case(30, 14, modvis=1, Twall=900.0, ktm=1, mix=_air()),
    "c01_512x256": lambda: euler_cosine_case(512, 256),
}
SCALARS = ("dt", "Href", "Cpref", "fm1D", "Fd1D", "Fpv1D", "Sg")
DEVICE_EXP = ("vlp", "vle", "vln", "kp", "ke", "kn")


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(STATE_CASES))
def test_initial_state_bitwise(name):
    case = STATE_CASES[name]()
    g, o = Simplec(case), OracleCase(case)
    try:
        for s in SCALARS:
            assert g.scalar(s) == o.scalar(s), s
        for f in NAMES + ["vin", "pina"]:
            a, b = g.field(f), o.field(f)
            assert a.shape == b.shape, f
            if case.ktm == 1 and f in DEVICE_EXP:
                assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), f
            else:
                assert np.array_equal(a, b), f
    finally:
        g.close()
