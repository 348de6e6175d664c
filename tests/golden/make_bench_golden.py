"""Regenerates tests/golden/bench_workloads.json from the CPU oracle: the
fixtures of the two Euler workloads the benchmark times.

* c01_euler_512x256_first20: the first 20 outer iterations of the C01 cosine
  nozzle at 512x256 real volumes (the benchmark's throughput workload), every
  report column and the itp_used of each iteration, plus checksums of the
  fields after iteration 20.
* c01_euler_80x40_converged: the C01 nozzle at 80x40 (the CPU-runnable case)
  run to the reference's stopping rule (normpl < tolt = 1e-10 first at it,
  stop at it_stop = 2 it; src/mach2d_main.f90:307,441-443): the stopping
  iteration, the converged integrals fmi, fme, Fd, fm1D and Cd = fme / fm1D
  (src/user/internal_flow/mod_intflow_postp.f90:1211), the wall pressure
  p(i, ny-1) (mod_intflow_postp.f90:430-445) and every 1000th report row.

Run: python tests/golden/make_bench_golden.py  (about a minute on one core)
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


def row(rep):
    return [rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd, rep.itp_used]


def first_iterations(case, n):
    o = OracleCase(case)
    hist = []
    for _ in range(n):
        rc, rep = o.iterate()
        if rc:
            raise RuntimeError(f"oracle stopped with rc={rc} at it={rep.it}")
        hist.append(row(rep))
    sums = {}
    for f in ("u", "v", "p", "T", "ro", "Uce", "Vcn", "roe", "ron"):
        a = o.field(f)
        sums[f] = {"sum": float(a.sum()), "abs_sum": float(abs(a).sum()), "max_abs": float(abs(a).max())}
    return {"case": case.as_dict(), "history_columns": COLS, "history": hist, "field_checksums": sums}


def converged(case, itmax=200000, every=1000):
    o = OracleCase(case)
    hist = []
    rep = None
    for _ in range(itmax):
        rc, rep = o.iterate()
        if rc:
            raise RuntimeError(f"oracle stopped with rc={rc} at it={rep.it}")
        if rep.it % every == 0:
            hist.append(row(rep))
        if o.scalar("it_stop") == rep.it:
            break
    p = o.field("p")
    nx, ny = o.nx, o.ny
    return {"case": case.as_dict(), "history_columns": COLS, "history_every": every, "history": hist,
            "final": {"it": rep.it, "it_stop": o.scalar("it_stop"), "normpl": rep.normpl, "fmi": rep.fmi,
                      "fme": rep.fme, "Fd": rep.Fd, "fm1D": o.scalar("fm1D"), "Cd": rep.fme / o.scalar("fm1D"),
                      "pwall": [p[(ny - 2) * nx + i] for i in range(nx)]}}


if __name__ == "__main__":
    out = {"c01_euler_512x256_first20": first_iterations(euler_cosine_case(512, 256), 20),
           "c01_euler_80x40_converged": converged(euler_cosine_case(80, 40))}
    path = os.path.join(HERE, "bench_workloads.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", path, "stop it", out["c01_euler_80x40_converged"]["final"]["it"])
