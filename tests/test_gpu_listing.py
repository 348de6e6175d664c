"""The reference's output files from the device run: the residual listing
(src/mach2d_main.f90:473-520) of the reference deck, row for row the same
text as the oracle's history formatted the same way, and the main-results
report (mod_intflow_postp.f90:1062-1256) of the converged run."""
import io

import pytest

from _oracle import OracleCase
from mach2d_b200.listing import ResidualListing, main_results
from mach2d_b200.simplec import Simplec, n01_case

pytestmark = pytest.mark.gpu


def test_listing_of_the_reference_deck():
    g = Simplec(n01_case())
    fh = io.StringIO()
    rep = g.run_listing(60, fh, wlf=10)
    lines = fh.getvalue().splitlines()
    assert lines[0] == ResidualListing.header()
    assert [int(ln[:10]) for ln in lines[1:]] == [10, 20, 30, 40, 50, 60, 60]
    o = OracleCase(n01_case())
    rows = []
    for _ in range(60):
        _, r = o.iterate()
        if r.it % 10 == 0:
            rows.append(ResidualListing.row(r))
    # the device run agrees with the oracle to 1e-9 relative: the 7-digit
    # columns of the listing are identical
    for a, b in zip(lines[1:7], rows):
        assert a[:70] == b[:70]
    assert rep.it == 60
    g.close()


def test_main_results_of_the_converged_reference_deck():
    c = n01_case()
    g = Simplec(c)
    g.set_graph(True)
    rep = g.run(3000)
    blocks, text = g.main_results(rep)
    o = OracleCase(c)
    for _ in range(rep.it):
        _, ro = o.iterate()
    f = {k: o.field(k) for k in ("x", "y", "re", "ye", "p", "roe", "u", "Uce")}
    ob, _ = main_results(o.nx, o.ny, f["x"], f["y"], f["re"], f["ye"], f["p"], f["roe"], f["u"], f["Uce"],
                         o.scalar("Sg"), c.Rc2, _ig(o.nx, o.ny, f["y"]), 1.4, c.p0,
                         o.scalar("Fpv1D"), o.scalar("Fd1D"), o.scalar("fm1D"), ro.fme)
    for k in blocks:
        for (a, _), (b, _) in zip(blocks[k], ob[k]):
            assert abs(a - b) <= 1e-6 * abs(b), k
    assert "*** Efficiency: numerical solution 2D / analytic Q1D (dimensionless) ***" in text
    g.close()


def _ig(nx, ny, y):
    for i in range(2, nx):
        if y[(ny - 2) * nx + i - 2] < y[(ny - 2) * nx + i - 1]:
            return i - 1
    return 1
