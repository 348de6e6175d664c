"""The reference's own Navier-Stokes deck (parametersNozzleNSPTV.txt with
geometry_n01.txt: N01 nozzle, 20x10, geometric clustering with a 1e-6 m
first cell, MIXTURE air, adiabatic wall) on the device, against the oracle's
run of it (tests/golden/ns_deck_n01.json, make_ns_deck.py): the same
stopping iteration, every 100th report to 1e-6 relative (the device exp/log
of mu and k and pow of the inlet differ from glibc in the last bits) and the
discharge coefficient to the 1e-6 of the integrals' specification."""
import json
import os

import pytest

from mach2d_b200.simplec import Case, Simplec

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "ns_deck_n01.json")


@pytest.mark.parametrize("graph", [False, True])
def test_reference_ns_deck_converges_like_the_oracle(graph):
    gold = json.load(open(GOLD))
    case = Case.from_dict(gold["case"])
    assert (case.modvis, case.ktm, case.kg, case.nxr, case.nyr) == (1, 1, 2, 20, 10)
    g = Simplec(case)
    g.set_graph(graph)
    rows = {r[0]: r for r in gold["every100"]}
    rep = None
    for it in range(1, 80001):
        rep = g.iterate()
        if it in rows:
            ref = rows[it]
            got = [rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd, rep.itp_used]
            assert got[8] == ref[8], it
            for k in (1, 5, 6, 7):
                assert abs(got[k] - ref[k]) <= 1e-6 * abs(ref[k]), (it, k)
        if g.scalar("it_stop") == rep.it:
            break
    assert rep.it == gold["final"][0]
    fmi, fme, Fd, Cd, _ = g.integrals()
    assert abs(Cd / gold["Cd"] - 1) < 1e-6
    assert abs(Fd / gold["final"][7] - 1) < 1e-6
    g.close()
