"""Gas-mixture thermophysical model (src/thermophysical/) behind the C ABI.

`Mixture` is the ctypes image of m2d_mixture; `mixture_init` mirrors
class_thermophysical_mixture%init (mod_class_thermophysical_mixture.f90:56-224)
on coefficient arrays; `read_species_database` reads the reference's
thermo_database.csv format (one block of ID_NAME / ID_M / ID_CPL / ID_CPU /
ID_VL / ID_VU / ID_KL / ID_KU rows per species) so that a user can pass the
reference's own data files.
"""
import ctypes

import numpy as np

from ._lib import check, lib

MAX_SPECIES = 8


class Mixture(ctypes.Structure):
    _fields_ = [("ngs", ctypes.c_int), ("Rg", ctypes.c_double),
                ("Xi", ctypes.c_double * MAX_SPECIES), ("Yi", ctypes.c_double * MAX_SPECIES),
                ("Mi", ctypes.c_double * MAX_SPECIES), ("Ri", ctypes.c_double * MAX_SPECIES),
                ("cpi", (ctypes.c_double * 10) * MAX_SPECIES),
                ("mui", (ctypes.c_double * 8) * MAX_SPECIES),
                ("kpi", (ctypes.c_double * 8) * MAX_SPECIES)]


def mixture_init(base, fractions, Mi, cpi, mui, kpi):
    """base 0: molar fractions, 1: mass fractions.  cpi (ngs, 10), mui and
    kpi (ngs, 8) in the database's coefficient order."""
    fr = np.ascontiguousarray(fractions, dtype=np.float64)
    n = fr.size
    arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (Mi, cpi, mui, kpi)]
    assert arrs[0].size == n and arrs[1].size == 10 * n and arrs[2].size == 8 * n and arrs[3].size == 8 * n
    m = Mixture()
    dp = ctypes.POINTER(ctypes.c_double)
    L = lib()
    L.m2d_mixture_init.argtypes = [ctypes.c_int, ctypes.c_int] + [dp] * 5 + [ctypes.POINTER(Mixture)]
    check(L.m2d_mixture_init(int(base), n, fr.ctypes.data_as(dp), *[a.ctypes.data_as(dp) for a in arrs],
                             ctypes.byref(m)))
    return m


def mixture_eval(m, T):
    """(cp, mu, kp, gm) of the mixture at temperature T (host evaluation)."""
    out = [ctypes.c_double() for _ in range(4)]
    L = lib()
    L.m2d_mixture_eval.argtypes = [ctypes.POINTER(Mixture), ctypes.c_double] + [ctypes.POINTER(ctypes.c_double)] * 4
    check(L.m2d_mixture_eval(ctypes.byref(m), float(T), *[ctypes.byref(v) for v in out]))
    return tuple(v.value for v in out)


def read_species_database(path, names):
    """Molar masses and coefficients of `names` from a file in the
    reference's thermo_database.csv format (one block per species, opened by
    ID_NAME and closed by END; text after the numbers of a row is a comment).
    Returns Mi (n,), cpi (n, 10), mui (n, 8), kpi (n, 8)."""
    def num(tok):
        return float(tok.replace("D", "E").replace("d", "e"))

    species, cur = {}, None
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts or not parts[0].startswith("ID_"):
                continue
            if parts[0] == "ID_NAME":
                cur = species.setdefault(parts[1], {})
                continue
            vals = []
            for t in parts[1:]:
                try:
                    vals.append(num(t))
                except ValueError:
                    break
            cur[parts[0]] = vals
    missing = [n for n in names if n not in species]
    if missing:
        raise KeyError(f"species not in {path}: {missing}")
    Mi = np.array([species[n]["ID_M"][0] for n in names])
    cpi = np.array([species[n]["ID_CPL"][:5] + species[n]["ID_CPU"][:5] for n in names])
    mui = np.array([species[n]["ID_VL"][:4] + species[n]["ID_VU"][:4] for n in names])
    kpi = np.array([species[n]["ID_KL"][:4] + species[n]["ID_KU"][:4] for n in names])
    return Mi, cpi, mui, kpi


def read_mixture_parameters(path):
    """(base, names, fractions) from a file in the reference's
    thermo_parameters.txt format: the base (0 molar, 1 mass) on the first
    line, then `fraction name` lines up to one named END
    (mod_class_thermophysical_mixture.f90:78-170)."""
    with open(path) as fh:
        lines = [ln.split() for ln in fh if ln.strip()]
    base = int(float(lines[0][0]))
    names, fr = [], []
    for parts in lines[1:]:
        if parts[1] == "END":
            break
        fr.append(float(parts[0].replace("D", "E").replace("d", "e")))
        names.append(parts[1])
    return base, names, fr


def mixture_from_files(parameters_path, database_path):
    """The MIXTURE model of class_thermophysical_mixture%init from its two
    input files; species whose fraction is <= 1e-8 are left out."""
    base, names, fr = read_mixture_parameters(parameters_path)
    keep = [k for k, f in enumerate(fr) if f > 1e-8]
    Mi, cpi, mui, kpi = read_species_database(database_path, [names[k] for k in keep])
    return mixture_init(base, [fr[k] for k in keep], Mi, cpi, mui, kpi)
