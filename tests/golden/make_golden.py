"""Regenerates the golden fixtures of tests/golden/ from the CPU oracle.

The reference cannot be run here (Fortran, no compiler in the image) and ships
no golden outputs, so these fixtures pin the oracle itself: the residual
history and the converged integrals of the reference's own Euler deck
(N01 nozzle, 20x10, mach2d_input/parametersNozzleEulerPTC.txt values) and of
the cosine-nozzle configuration at 40x20.  Run: python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from _oracle import OracleCase  # noqa: E402
from mach2d_b200.simplec import euler_cosine_case, n01_case  # noqa: E402


def run(case, itmax, keep=40):
    o = OracleCase(case)
    hist = []
    rep = None
    for k in range(itmax):
        rc, rep = o.iterate()
        if rc:
            raise RuntimeError(f"oracle stopped with rc={rc} at it={rep.it}")
        if k < keep:
            hist.append([rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd,
                         rep.itp_used])
        if o.scalar("it_stop") == rep.it:
            break
    p = o.field("p")
    nx, ny = o.nx, o.ny
    pwall = [p[(ny - 2) * nx + i] for i in range(nx)]
    return {
        "case": case.as_dict(),
        "history_columns": ["it", "dt", "norm", "normpl", "rmass", "fmi", "fme", "Fd", "itp_used"],
        "history": hist,
        "final": {"it": rep.it, "it_stop": o.scalar("it_stop"), "normpl": rep.normpl,
                  "fmi": rep.fmi, "fme": rep.fme, "Fd": rep.Fd, "fm1D": o.scalar("fm1D"),
                  "Cd": rep.fme / o.scalar("fm1D"), "pwall": pwall},
    }


if __name__ == "__main__":
    out = {"n01_euler_20x10": run(n01_case(), 3000),
           "c01_euler_40x20_first60": run(euler_cosine_case(40, 20), 60, keep=60)}
    with open(os.path.join(HERE, "oracle_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", os.path.join(HERE, "oracle_golden.json"))
