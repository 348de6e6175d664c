"""Writes the oracle's residual history of the Navier-Stokes nozzle with the
MIXTURE model (air from air_species.json) at 512 x 256 real volumes (C01
cosine nozzle, geometric wall clustering with a first cell of 1e-6 m,
p0 = 2 MPa, T0 = 1500 K, adiabatic wall, FP64 MSI): every 25th iteration
and the iteration at which the run stops with a NaN.

    python tests/golden/make_ns512_trace.py          laminar -> ns512_mixture_trace.json
    python tests/golden/make_ns512_trace.py bl       Baldwin-Lomax eddy viscosity (modtur = 1,
                                                     Pr_t = 0.9) -> ns512_bl_mixture_trace.json

About four minutes of one CPU core each.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from _oracle import OracleCase  # noqa: E402
from mach2d_b200.simplec import euler_cosine_case  # noqa: E402
from mach2d_b200.thermo import mixture_init  # noqa: E402


def ns512_case(solver=0, modtur=0):
    d = json.load(open(os.path.join(HERE, "air_species.json")))
    mix = mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])
    return euler_cosine_case(512, 256, modvis=1, kg=2, a1=1e-6, p0=2e6, T0=1500.0, Twall=-1.0, ktm=1, mix=mix,
                             solver=solver, modtur=modtur, prt=0.9)


def main(bl=False):
    o = OracleCase(ns512_case(modtur=1 if bl else 0))
    rows, stop = [], None
    for it in range(1, 3001):
        rc, rep = o.iterate()
        if rc != 0 or not np.isfinite(rep.norm):
            stop = it
            break
        if it % 25 == 0:
            rows.append([rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd, rep.itp_used])
    out = {"columns": ["it", "dt", "norm", "normpl", "rmass", "fmi", "fme", "Fd", "itp_used"], "every25": rows,
           "nan_at": stop}
    name = "ns512_bl_mixture_trace.json" if bl else "ns512_mixture_trace.json"
    with open(os.path.join(HERE, name), "w") as fh:
        json.dump(out, fh)


if __name__ == "__main__":
    main(bl=len(sys.argv) > 1 and sys.argv[1] == "bl")
