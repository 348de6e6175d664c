"""Reader for MACH-2D input decks (src/util/class_ifile.f90:50-112).

A data line is `value & name & description`; any other line is a comment.
`case_from_decks` maps a parameters deck plus a geometry deck onto the
m2d_case of the device-resident iteration (src/mod_mach2d_data.f90:186-233,
src/grid/mod_grid.f90:44-75, src/solvers/mod_solvers.f90:17-87,
src/tstepper/mod_tstepper*.f90, src/thermophysical/mod_thermophysical.f90:20-75).
"""
import os

from .simplec import Case
from .thermo import mixture_from_files


def parse(path, delimiter="&"):
    values = {}
    with open(path) as fh:
        for line in fh:
            parts = line.split(delimiter)
            if len(parts) < 3:
                continue
            val, name = parts[0].strip(), parts[1].strip()
            if name:
                values[name] = val
    return values


def fnum(s):
    return float(s.replace("d", "e").replace("D", "e"))


def _resolve(path, base_dir):
    """A deck names its data files relative to the directory the solver runs
    in (./mach2d_input/...): try the current directory, then base_dir."""
    if os.path.isabs(path) or os.path.exists(path):
        return path
    return os.path.join(base_dir, path)


def case_from_decks(params_path, geometry_path, base_dir=None):
    """base_dir: where the deck's relative data-file paths start (default:
    the parent of the deck's own directory)."""
    p = parse(params_path)
    g = parse(geometry_path)
    if base_dir is None:
        base_dir = os.path.dirname(os.path.dirname(os.path.abspath(params_path)))
    model = p.get("thermo_model", "").strip()
    if model not in ("CONSTANT", "MIXTURE"):
        raise ValueError(f"thermophysical_initialization: Unknown opton: {model}")
    if int(p["kflow"]) != 1:
        raise ValueError("only internal flow (kflow = 1) is supported")
    nmf, nmd = int(p["nmf"]), int(p["nmd"])
    scale = 2 ** (nmd - 1)
    c = Case()
    gid = g["ID"].strip()
    if gid == "N01":
        c.geom = 1
        for k in ("Rth", "Rin", "Rout", "Rc1", "Rc2", "Rc3", "alf", "bet", "Lchamb"):
            setattr(c, k, fnum(g[k]))
    elif gid == "C01":
        c.geom = 0
        for k in ("Lc", "Ld", "Rin", "Rout"):
            setattr(c, k, fnum(g[k]))
    else:
        raise ValueError(f"unknown geometry ID {gid}")
    del nmf
    c.nxr = int(p["nxi-2"]) * scale
    c.nyr = int(p["nyi-2"]) * scale
    c.kg, c.kcm, c.a1 = int(p["kg"]), int(p["kcm"]), fnum(p["a1"])
    c.coord, c.modvis, c.beta = int(p["coord"]), int(p["modvis"]), fnum(p["beta"])
    c.p0, c.T0, c.Twall = fnum(p["P0"]), fnum(p["T0"]), fnum(p["Tnbc"])
    c.Rg, c.gamma = fnum(p["thermo_const_Rg"]), fnum(p["thermo_const_gamma"])
    c.mu, c.kappa = fnum(p["thermo_const_mu"]), fnum(p["thermo_const_kappa"])
    c.itmmax, c.itpmax = int(p["itmmax"]), int(p["itpmax"])
    c.tolm, c.tolt = fnum(p["tolm"]), fnum(p["tolt"])
    ks = p["solver"].strip()
    if ks not in ("MSI", "TDMA"):
        raise ValueError(f"solvers_init: Unkown option: {ks}")
    c.solver = 0 if ks == "MSI" else 1
    c.nitm_u, c.nitm_p = int(p["nitm_u"]), int(p["nitm_p"])
    c.tol_u, c.tol_p = fnum(p["tol_u"]), fnum(p["tol_p"])
    dm = p["dtmodel"].strip()
    if dm not in ("RAMP", "SCARBOROUGH"):
        raise ValueError(f"tstepper_init: Unknown model: {dm}")
    c.dtmodel = 0 if dm == "RAMP" else 1
    c.dt1, c.dt2 = fnum(p["dt1"]), fnum(p["dt2"])
    c.it1, c.it2 = int(p["it1"]), int(p["it2"])
    c.h0, c.mincc, c.maxcc = fnum(p["h0"]), fnum(p["mincc"]), fnum(p["maxcc"])
    c.nan_policy = 0
    c.ktm = 0
    if model == "MIXTURE":
        c.ktm = 1
        c.mix = mixture_from_files(_resolve(p["thermo_mix_parameters"].strip(), base_dir),
                                   _resolve(p["thermo_mix_database"].strip(), base_dir))
    return c
