"""Writes ns_deck_n01.json: the reference's own Navier-Stokes deck
(mach2d_input/parametersNozzleNSPTV.txt with geometry_n01.txt: N01 nozzle
at 20x10, geometric wall clustering with a 1e-6 m first cell, MIXTURE air,
adiabatic wall, FP64 MSI) run by the oracle to its stopping iteration: the
case as read by mach2d_b200.ifile, every 100th report and the final
integrals.

    python tests/golden/make_ns_deck.py <path of the reference checkout>
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from _oracle import OracleCase  # noqa: E402
from mach2d_b200.ifile import case_from_decks  # noqa: E402


def main(ref):
    inp = os.path.join(ref, "mach2d_input")
    c = case_from_decks(os.path.join(inp, "parametersNozzleNSPTV.txt"), os.path.join(inp, "geometry_n01.txt"),
                        base_dir=ref)
    o = OracleCase(c)
    rows = []
    for it in range(1, 80001):
        rc, r = o.iterate()
        if rc:
            raise RuntimeError(f"oracle stopped with {rc} at {it}")
        row = [r.it, r.dt, r.norm, r.normpl, r.rmass, r.fmi, r.fme, r.Fd, r.itp_used]
        if it % 100 == 0:
            rows.append(row)
        if o.scalar("it_stop") == r.it:
            break
    out = {"case": c.as_dict(), "every100": rows, "final": row, "fm1D": o.scalar("fm1D"),
           "Cd": r.fme / o.scalar("fm1D")}
    with open(os.path.join(HERE, "ns_deck_n01.json"), "w") as fh:
        json.dump(out, fh)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
