"""The reference's output files written by mach2d_b200.listing: Fortran edit
descriptors, the residual listing of src/mach2d_main.f90:473-520 and the
main-results report of mod_intflow_postp.f90:1062-1256, checked on the
oracle's converged N01 run."""
import json
import math
import os

import numpy as np

from _oracle import OracleCase
from mach2d_b200.listing import ResidualListing, fortran_a, fortran_es, main_results
from mach2d_b200.simplec import Report, n01_case

GOLD = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.json")


def test_edit_descriptors():
    assert fortran_es(1.0, 14, 7) == " 1.0000000E+00"
    assert fortran_es(-1.2345678e-3, 14, 7) == "-1.2345678E-03"
    assert fortran_es(0.0, 14, 7) == " 0.0000000E+00"
    assert fortran_es(1e-100, 14, 7) == " 1.0000000-100"
    assert fortran_es(9.99999999e5, 14, 7) == " 1.0000000E+06"
    assert fortran_es(12345.678901234567, 25, 15) == "    1.234567890123457E+04"
    assert fortran_es(float("nan"), 14, 7) == "           NaN"
    assert fortran_a("max(|pl|)/p_avg", 14) == "max(|pl|)/p_av"      # A14 keeps the leftmost 14
    assert fortran_a("it", 10) == "        it"


def test_residual_listing_rows():
    h = ResidualListing.header()
    assert h.startswith("        it             dt           norm max(|pl|)/p_av          rmass")
    assert h.endswith("                    fmi                 fme/fmi                      Fd")
    r = Report(it=7, dt=2.5e-6, norm=1.25e-3, normpl=3.0e-4, rmass=4.5e-9, fmi=10.0, fme=5.0, Fd=123.0, itp_used=2)
    row = ResidualListing.row(r)
    assert row == ("         7  2.5000000E-06  1.2500000E-03  3.0000000E-04  4.5000000E-09"
                   "  1.0000000000000000E+01  5.0000000000000000E-01  1.2300000000000000E+02")

    class F:
        def __init__(self):
            self.s = ""

        def write(self, t):
            self.s += t
    f = F()
    lst = ResidualListing(f, wlf=5)
    for it in range(1, 8):
        r.it = it
        lst.write(r, finished=(it == 7))
    assert f.s.count("\n") == 3 and f.s.splitlines()[1].startswith("         5")


def test_main_results_on_the_converged_reference_deck():
    gold = json.load(open(GOLD))["n01_euler_20x10"]["final"]
    case = n01_case()
    o = OracleCase(case)
    for _ in range(gold["it"]):
        rc, rep = o.iterate()
    nx, ny = o.nx, o.ny
    fld = {k: o.field(k) for k in ("x", "y", "re", "ye", "p", "roe", "u", "Uce")}
    y = fld["y"]
    ig = 1
    for i in range(2, nx):
        if y[(ny - 2) * nx + i - 2] < y[(ny - 2) * nx + i - 1]:
            ig = i - 1
            break
    blocks, text = main_results(nx, ny, fld["x"], y, fld["re"], fld["ye"], fld["p"], fld["roe"], fld["u"],
                                fld["Uce"], o.scalar("Sg"), case.Rc2, ig, case.gamma, case.p0, o.scalar("Fpv1D"),
                                o.scalar("Fd1D"), o.scalar("fm1D"), rep.fme)
    assert blocks["efficiency"][0][0] == gold["Cd"]
    # the report's dynamic thrust takes u of the ghost column; the residual
    # listing's (get_mass_flow_rate_and_thrust) the face mean: close, not equal
    assert abs(blocks["numeric"][1][0] / rep.Fd - 1) < 0.05
    assert 0.9 < blocks["kl"][0][0] < 1.0
    assert all(math.isfinite(v) for blk in blocks.values() for v, _ in blk)
    lines = text.splitlines()
    assert lines[1] == " *** Analytic solution of the Q1D isentropic flow ***"
    assert len(lines) == 3 + 14 + 3 + 1 + 3 + 14 + 3 + 13
    assert lines[3].endswith(" = fm1D:  mass flow rate (kg/s)") and len(lines[3].split(" = ")[0]) == 25
    assert np.isclose(float(lines[-13].split(" = ")[0]), gold["Cd"], rtol=1e-14)
