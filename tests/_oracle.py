"""ctypes binding of the CPU oracle (oracle/liboracle.so), used by the tests as
the checker.  Builds the oracle with make when the shared object is missing."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.orc_create.restype = ctypes.c_void_p
        _lib.orc_scalar.restype = ctypes.c_double
        _lib.orc_scalar.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        _lib.orc_field.restype = ctypes.c_long
        _lib.orc_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                   ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        for fn in ("orc_norm_l1_5d", "orc_norm_l1_9d", "orc_norm_l1_9d_relative", "orc_norm_l1_b",
                   "orc_check_mass_conservation", "orc_get_isentropic_mass_flow",
                   "orc_get_mach_area", "orc_get_gp_ratio", "orc_tstepper_dt0_scarborough",
                   "orc_get_mean_cc_9d", "orc_get_mean_cc_5d", "orc_tstepper_dt_scarborough"):
            getattr(_lib, fn).restype = ctypes.c_double
    return _lib


def _conv(args):
    out = []
    for a in args:
        if isinstance(a, np.ndarray):
            assert a.dtype == np.float64 and a.flags.c_contiguous
            out.append(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        elif isinstance(a, (bool, int, np.integer)):
            out.append(ctypes.c_int(int(a)))
        elif isinstance(a, (float, np.floating)):
            out.append(ctypes.c_double(float(a)))
        else:
            out.append(a)
    return out


def call(name, *args):
    """Calls orc_<name> with by-value scalars and numpy arrays."""
    return getattr(lib(), "orc_" + name)(*_conv(args))


class OracleCase:
    """Full oracle state of one nozzle instance (oracle/driver.c)."""

    def __init__(self, case):
        from mach2d_b200.simplec import Case  # layout shared with the C ABI struct
        assert isinstance(case, Case)
        self._case = case
        self.s = ctypes.c_void_p(lib().orc_create(ctypes.byref(case)))
        self.nx = lib().orc_nx(self.s)
        self.ny = lib().orc_ny(self.s)

    def __del__(self):
        try:
            lib().orc_destroy(self.s)
        except Exception:
            pass

    def iterate(self):
        from mach2d_b200.simplec import Report
        rep = Report()
        rc = lib().orc_iterate(self.s, ctypes.byref(rep))
        return rc, rep

    def field(self, name):
        p = ctypes.POINTER(ctypes.c_double)()
        n = lib().orc_field(self.s, name.encode(), ctypes.byref(p))
        if n < 0:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def scalar(self, name):
        return lib().orc_scalar(self.s, name.encode())
