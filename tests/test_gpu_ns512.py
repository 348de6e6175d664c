"""Navier-Stokes with the MIXTURE model at 512 x 256 against the oracle's
history (tests/golden/ns512_mixture_trace.json, make_ns512_trace.py).

The C01 nozzle with geometric wall clustering (first cell 1e-6 m), air,
p0 = 2 MPa, T0 = 1500 K and an adiabatic wall, FP64 MSI: every 25th
iteration's report columns agree with the oracle's to 1e-6 relative (the
inlet pow() and the device exp/log of mu and k differ from glibc in the
last bit, and the run amplifies such differences slowly), the p' cycle
counts agree exactly, and the run stops with a NaN at the same iteration as
the oracle's: the Scarborough time step grows past what the scheme
tolerates, a property of the algorithm that both implementations share.
The same holds with the Baldwin-Lomax eddy viscosity wired in (modtur = 1,
Pr_t = 0.9; fixture ns512_bl_mixture_trace.json): the configuration the
turbulent 512 x 256 case specifies.
"""
import json
import os

import pytest

from mach2d_b200 import M2DError
from mach2d_b200.simplec import Simplec, euler_cosine_case
from mach2d_b200.thermo import mixture_init

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _case(modtur):
    d = json.load(open(os.path.join(GOLD, "air_species.json")))
    mix = mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])
    return euler_cosine_case(512, 256, modvis=1, kg=2, a1=1e-6, p0=2e6, T0=1500.0, Twall=-1.0, ktm=1, mix=mix,
                             solver=0, modtur=modtur, prt=0.9)


@pytest.mark.parametrize("modtur,trace", [(0, "ns512_mixture_trace.json"), (1, "ns512_bl_mixture_trace.json")])
def test_ns512_mixture_history_matches_oracle(modtur, trace):
    gold = json.load(open(os.path.join(GOLD, trace)))
    rows = {r[0]: r for r in gold["every25"]}
    g = Simplec(_case(modtur))
    stop = None
    for it in range(1, gold["nan_at"] + 1 if gold["nan_at"] else 3001):
        try:
            rep = g.iterate()
        except M2DError as e:
            assert e.code == 3
            stop = it
            break
        if it in rows:
            ref = rows[it]
            got = [rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd, rep.itp_used]
            assert got[8] == ref[8], it
            for k in range(1, 8):
                assert abs(got[k] - ref[k]) <= 1e-6 * abs(ref[k]) + 1e-300, (it, gold["columns"][k])
    assert stop == gold["nan_at"]
    g.close()
