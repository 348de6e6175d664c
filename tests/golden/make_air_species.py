"""Writes air_species.json: the species data of the reference's default
MIXTURE deck (mach2d_input/thermo_parameters.txt, molar fractions Ar 0.01,
N2 0.78, O2 0.21) read from its mach2d_input/thermo_database.csv with the
package's own parsers, so that the GPU tests can build that mixture without
the reference tree.

    python tests/golden/make_air_species.py <path of the reference checkout>
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mach2d_b200.thermo import read_mixture_parameters, read_species_database  # noqa: E402


def main(ref):
    inp = os.path.join(ref, "mach2d_input")
    base, names, fr = read_mixture_parameters(os.path.join(inp, "thermo_parameters.txt"))
    keep = [k for k, f in enumerate(fr) if f > 1e-8]
    names = [names[k] for k in keep]
    Mi, cpi, mui, kpi = read_species_database(os.path.join(inp, "thermo_database.csv"), names)
    out = {"base": base, "names": names, "fractions": [fr[k] for k in keep], "Mi": Mi.tolist(),
           "cpi": cpi.tolist(), "mui": mui.tolist(), "kpi": kpi.tolist()}
    with open(os.path.join(HERE, "air_species.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
