"""CPU-side checks of the C ABI: the library loads without a GPU, exports
every entry point include/mach2d_b200.h declares, rejects bad arguments
without touching the device, and the host-side mirrors behave like the
reference's (solver factory, deck reader)."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import mach2d_b200
from mach2d_b200 import _lib
from mach2d_b200.solvers import solvers_init

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.exported_symbols()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    nm = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert f" T {n}\n" in nm + "\n", n


def test_bad_arguments_are_rejected_before_any_device_work():
    nx = ctypes.c_int(2)
    ny = ctypes.c_int(5)
    nitm = ctypes.c_int(5)
    tol = ctypes.c_double(1e-2)
    L = _lib.lib()
    buf = (ctypes.c_double * 90)()
    rc = L.m2d_msi9_solve(ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nitm), ctypes.byref(tol),
                          buf, buf, buf)
    assert rc == 2
    assert b"bad arguments" in L.m2d_last_error()
    big = ctypes.c_int(100000)
    ok = ctypes.c_int(10)
    rc = L.m2d_msi5_solve(ctypes.byref(ok), ctypes.byref(big), ctypes.byref(nitm), ctypes.byref(tol),
                          buf, buf, buf)
    assert rc in (2, 6)


def test_wait_hook_rejects_bad_arguments():
    # the failure-detection test hook only sets host state; it is exercised on
    # the GPU by test_gpu_wait_timeout.py
    L = _lib.lib()
    L.m2d_test_wait_hook.argtypes = [ctypes.c_int, ctypes.c_double]
    assert L.m2d_test_wait_hook(3, 0.01) == 2
    assert L.m2d_test_wait_hook(1, 20.0) == 2
    assert L.m2d_test_wait_hook(1, -1.0) == 2
    assert L.m2d_test_wait_hook(0, 0.0) == 0


def test_msi_max_ny_fits_shared_memory():
    assert _lib.lib().m2d_msi_max_ny() >= 1026


def test_solvers_init_mirrors_reference_factory():
    s5, s9 = solvers_init(10, 8, "MSI", 5, 20, 1e-2, 1e-2)
    assert (s5.nitm, s9.nitm, s5.ndiag, s9.ndiag) == (20, 5, 5, 9)
    s5, s9 = solvers_init(10, 8, "TDMA ", 3, 4, 0, 0)
    assert type(s9).__name__ == "ClassSolverTDMA9d"
    with pytest.raises(ValueError):
        solvers_init(10, 8, "CG", 1, 1, 0, 0)


def test_array_arguments_are_type_checked():
    with pytest.raises(TypeError):
        _lib.dptr(np.zeros(4, dtype=np.float32))
    with pytest.raises(TypeError):
        _lib.dptr(np.zeros((4, 4))[:, 1])


def test_deck_reader_maps_a_reference_style_deck(tmp_path):
    from mach2d_b200.ifile import case_from_decks, parse
    deck = os.path.join(ROOT, "tests", "golden", "deck_euler_n01.txt")
    geom = os.path.join(ROOT, "tests", "golden", "geometry_n01.txt")
    c = case_from_decks(deck, geom)
    assert (c.geom, c.nxr, c.nyr, c.modvis, c.solver, c.dtmodel) == (1, 20, 10, 0, 0, 1)
    assert c.Rth == pytest.approx(2.29108e-2)
    assert parse(deck)["sim_id"] == "n01"


def test_package_points_at_in_tree_library():
    assert os.path.dirname(mach2d_b200.LIB_PATH) == os.path.join(ROOT, "mach2d_b200")


REF_INPUT = "/root/reference/mach2d_input"


@pytest.mark.skipif(not os.path.isdir(REF_INPUT), reason="reference input decks not present")
def test_deck_reader_builds_the_mixture_of_a_reference_mixture_deck():
    """parametersNozzleNSPTV.txt selects thermo_model = MIXTURE; its species
    come from thermo_parameters.txt and thermo_database.csv."""
    from mach2d_b200.ifile import case_from_decks
    from mach2d_b200.thermo import mixture_init
    c = case_from_decks(os.path.join(REF_INPUT, "parametersNozzleNSPTV.txt"),
                        os.path.join(REF_INPUT, "geometry_n01.txt"), base_dir=os.path.dirname(REF_INPUT))
    assert (c.ktm, c.modvis, c.mix.ngs) == (1, 1, 3)
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "air_species.json")))
    m = mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])
    assert bytes(m) == bytes(c.mix)


def test_air_fixture_gives_air_properties():
    from mach2d_b200.thermo import mixture_eval, mixture_init
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "air_species.json")))
    m = mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])
    cp, mu, kp, gm = mixture_eval(m, 300.0)
    assert m.Rg == pytest.approx(287.0, rel=1e-4)
    assert cp == pytest.approx(1004.5, rel=2e-3) and gm == pytest.approx(1.400, rel=1e-3)
    assert mu == pytest.approx(1.85e-5, rel=2e-2) and kp == pytest.approx(0.0262, rel=3e-2)


def test_extrapolation_rejects_bad_sizes_before_any_device_work():
    z = np.zeros(8)
    for nx, ny, itemax in ((4, 20000, 1), (3, 8, 1), (8, 8, -1)):
        with pytest.raises(_lib.M2DError) as e:
            _lib.call("m2d_extflow_extrapolate_ro_to_fictitious", nx, ny, itemax, 1.0, z, z, z, z, z)
        assert e.value.code == 2
