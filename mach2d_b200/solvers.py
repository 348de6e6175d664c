"""Linear-solver plug-ins with the interface of src/solvers/.

`solvers_init` mirrors src/solvers/mod_solvers.f90:17-87 (selection by
"MSI" / "TDMA", unknown option is an error; "MSI_MIXED" is this library's
FP32-sweep variant); each class mirrors
class_solver_*%init / %solve (src/solvers/mod_solver_msi.f90,
mod_solver_tdma.f90).  `solve(a, b, sol)` updates `sol` in place like the
Fortran `intent(inout)` argument.  a is a (k, nx*ny) float64 array whose row
k-1 is diagonal k of the reference's a(nx*ny, k).
"""
import numpy as np

from ._lib import call


class ClassSolverMSI9d:
    """class_solver_msi9d (src/solvers/mod_solver_msi.f90:96-133)."""

    ndiag = 9

    def init(self, nx, ny, nitm, tol):
        self.nx, self.ny, self.nitm, self.tol = int(nx), int(ny), int(nitm), float(tol)
        self.nit = 0
        return self

    def solve(self, a, b, sol):
        import ctypes
        nit = ctypes.c_int(0)
        call("m2d_msi9_solve_it" if self.ndiag == 9 else "m2d_msi5_solve_it",
             self.nx, self.ny, self.nitm, self.tol, _mat(a, self.ndiag, self.nx * self.ny),
             _vec(b), _vec(sol), nit)
        self.nit = nit.value


class ClassSolverMSI5d(ClassSolverMSI9d):
    """class_solver_msi5d (src/solvers/mod_solver_msi.f90:56-93)."""

    ndiag = 5


class ClassSolverMSIMixed9d(ClassSolverMSI9d):
    """No counterpart in the reference: MSI whose factorisation and sweeps run
    in FP32 inside the FP64 iteration (m2d_msi9_solve_mixed)."""

    def solve(self, a, b, sol):
        import ctypes
        nit = ctypes.c_int(0)
        call("m2d_msi9_solve_mixed" if self.ndiag == 9 else "m2d_msi5_solve_mixed",
             self.nx, self.ny, self.nitm, self.tol, _mat(a, self.ndiag, self.nx * self.ny),
             _vec(b), _vec(sol), nit)
        self.nit = nit.value


class ClassSolverMSIMixed5d(ClassSolverMSIMixed9d):
    ndiag = 5


class ClassSolverTDMA9d:
    """class_solver_tdma9d (src/solvers/mod_solver_tdma.f90:76-100)."""

    ndiag = 9

    def init(self, nx, ny, nitm):
        self.nx, self.ny, self.nitm = int(nx), int(ny), int(nitm)
        return self

    def solve(self, a, b, sol):
        call("m2d_tdma9_solve" if self.ndiag == 9 else "m2d_tdma5_solve",
             self.nx, self.ny, self.nitm, _mat(a, self.ndiag, self.nx * self.ny), _vec(b), _vec(sol))


class ClassSolverTDMA5d(ClassSolverTDMA9d):
    """class_solver_tdma5d (src/solvers/mod_solver_tdma.f90:48-72)."""

    ndiag = 5


def solvers_init(nx, ny, ksolver, nitm_u, nitm_p, tol_u, tol_p):
    """Returns (solver5d, solver9d) as src/solvers/mod_solvers.f90:17-87."""
    k = ksolver.strip()
    if k == "MSI":
        return (ClassSolverMSI5d().init(nx, ny, nitm_p, tol_p),
                ClassSolverMSI9d().init(nx, ny, nitm_u, tol_u))
    if k == "TDMA":
        return ClassSolverTDMA5d().init(nx, ny, nitm_p), ClassSolverTDMA9d().init(nx, ny, nitm_u)
    if k == "MSI_MIXED":
        return (ClassSolverMSIMixed5d().init(nx, ny, nitm_p, tol_p),
                ClassSolverMSIMixed9d().init(nx, ny, nitm_u, tol_u))
    raise ValueError(f"solvers_init: Unkown option: {k}")


def norm_l1_5d(nx, ny, var, b, a, norm):
    """src/solvers/mod_solvers.f90:91-125; returns the updated norm."""
    import ctypes
    n = ctypes.c_double(norm)
    call("m2d_norm_l1_5d", nx, ny, _vec(var), _vec(b), _mat(a, 5, nx * ny), n)
    return n.value


def norm_l1_9d(nx, ny, var, b, a, norm):
    """src/solvers/mod_solvers.f90:128-170."""
    import ctypes
    n = ctypes.c_double(norm)
    call("m2d_norm_l1_9d", nx, ny, _vec(var), _vec(b), _mat(a, 9, nx * ny), n)
    return n.value


def norm_l1_9d_relative(nx, ny, var, b, a, norm):
    """src/solvers/mod_solvers.f90:176-245."""
    import ctypes
    n = ctypes.c_double(norm)
    call("m2d_norm_l1_9d_relative", nx, ny, _vec(var), _vec(b), _mat(a, 9, nx * ny), n)
    return n.value


def tdma_lines(aw, ap, ae, d):
    """Independent tridiagonal lines, arrays of shape (nlines, n)."""
    nlines, n = ap.shape
    x = np.zeros_like(ap)
    call("m2d_tdma_lines", n, nlines, _vec(aw), _vec(ap), _vec(ae), _vec(d), x)
    return x


def _vec(v):
    if not (isinstance(v, np.ndarray) and v.dtype == np.float64 and v.flags.c_contiguous):
        raise TypeError("arrays must be C-contiguous float64")
    return v


def _mat(a, k, n):
    a = _vec(a)
    if a.size != k * n:
        raise ValueError(f"coefficient array must hold {k} planes of {n}")
    return a


class FgmresReport:
    """m2d_fgmres_report of include/mach2d_b200.h."""

    def __init__(self, raw):
        for k in ("iterations", "msi_applications", "learned_applications", "cycles", "converged", "rel_residual"):
            setattr(self, k, getattr(raw, k))


def fgmres(nd, nx, ny, a, b, x, tol, prec=0, restart=30, maxit=1000, net=None, Jp=None, work=None, stream=None):
    """Flexible GMRES with the MSI factorisation (prec 0 FP64, 1 FP32) or the
    learned correction plus one FP32 MSI step (prec 2, nd = 5) as its
    preconditioner (m2d_fgmres_solve).  a, b, x, Jp: CUDA float64 tensors in
    the reference layout; x is updated in place.  Returns an FgmresReport;
    raises M2DError unless |b - A x| <= tol |b| within maxit steps."""
    import ctypes

    import torch

    from ._lib import check, lib

    class _Rep(ctypes.Structure):
        _fields_ = [("iterations", ctypes.c_int), ("msi_applications", ctypes.c_int),
                    ("learned_applications", ctypes.c_int), ("cycles", ctypes.c_int), ("converged", ctypes.c_int),
                    ("rel_residual", ctypes.c_double)]

    L = lib()
    L.m2d_fgmres_workspace_doubles.restype = ctypes.c_long
    L.m2d_fgmres_workspace_doubles.argtypes = [ctypes.c_int] * 4
    L.m2d_fgmres_solve.argtypes = ([ctypes.c_int] * 5 + [ctypes.c_double] + [ctypes.c_void_p] * 3 + [ctypes.c_int]
                                   + [ctypes.c_void_p] * 4 + [ctypes.POINTER(_Rep)])
    if work is None:
        work = torch.empty(L.m2d_fgmres_workspace_doubles(nd, nx, ny, restart), dtype=torch.float64,
                           device=x.device)
    rep = _Rep()
    check(L.m2d_fgmres_solve(nd, nx, ny, restart, maxit, tol, a.data_ptr(), b.data_ptr(), x.data_ptr(), prec,
                             None if net is None else net._h, None if Jp is None else Jp.data_ptr(),
                             work.data_ptr(), stream, ctypes.byref(rep)))
    return FgmresReport(rep)
