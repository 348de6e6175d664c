"""Writes ttr512_c01_euler.json: the oracle's run of the C01 cosine nozzle
at 512x256 real volumes (Euler, constant properties, FP64 MSI, SCARBOROUGH)
with tolt = 1e-8, the reference's stopping rule (normpl < tolt first at it,
stop at it_stop = 2 it; src/mach2d_main.f90:307,441-443).  It records every
1000th report row and the integrals -- fmi, fme, Fd, Cd = fme / fm1D
(src/user/internal_flow/mod_intflow_postp.f90:1211) and the wall pressure
p(i, ny-1) (mod_intflow_postp.f90:430-445) -- at the first iteration with
normpl < 1e-8 ("first_below") and at the stopping iteration ("final").  The
file is rewritten every 5000 iterations, so a partial run leaves the rows so
far.  About 200,000 iterations: several hours of one CPU core.

    python tests/golden/make_ttr512_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from _oracle import OracleCase  # noqa: E402
from mach2d_b200.simplec import euler_cosine_case  # noqa: E402

COLS = ["it", "dt", "norm", "normpl", "rmass", "fmi", "fme", "Fd", "itp_used"]
OUT = os.path.join(HERE, "ttr512_c01_euler.json")


def integrals(o, rep):
    p = o.field("p")
    nx, ny = o.nx, o.ny
    return {"it": rep.it, "normpl": rep.normpl, "fmi": rep.fmi, "fme": rep.fme, "Fd": rep.Fd,
            "fm1D": o.scalar("fm1D"), "Cd": rep.fme / o.scalar("fm1D"),
            "pwall": [p[(ny - 2) * nx + i] for i in range(nx)]}


def main(itmax=400000):
    case = euler_cosine_case(512, 256, tolt=1e-8)
    o = OracleCase(case)
    out = {"case": case.as_dict(), "history_columns": COLS, "history_every": 1000, "history": [],
           "first_below": None, "final": None, "complete": False}
    for _ in range(itmax):
        rc, rep = o.iterate()
        if rc:
            raise RuntimeError(f"oracle stopped with rc={rc} at it={rep.it}")
        if rep.it % 1000 == 0:
            out["history"].append([rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd,
                                   rep.itp_used])
        if out["first_below"] is None and rep.normpl < 1e-8:
            out["first_below"] = integrals(o, rep)
            json.dump(out, open(OUT, "w"))
        if o.scalar("it_stop") == rep.it:
            out["final"] = integrals(o, rep)
            out["complete"] = True
            break
        if rep.it % 5000 == 0:
            json.dump(out, open(OUT, "w"))
    json.dump(out, open(OUT, "w"))


if __name__ == "__main__":
    main()
