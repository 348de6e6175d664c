"""Device-resident SIMPLEC driver: the set-up and `it` loop of
src/mach2d_main.f90:25-445 for internal flow, run through the C ABI context
(m2d_create / m2d_iterate / m2d_run)."""
import ctypes

import numpy as np

from ._lib import check, lib
from .thermo import Mixture


class Case(ctypes.Structure):
    """m2d_case of include/mach2d_b200.h (one nozzle instance)."""

    _fields_ = [
        ("geom", ctypes.c_int), ("Lc", ctypes.c_double), ("Ld", ctypes.c_double),
        ("Rin", ctypes.c_double), ("Rout", ctypes.c_double), ("Rth", ctypes.c_double),
        ("Rc1", ctypes.c_double), ("Rc2", ctypes.c_double), ("Rc3", ctypes.c_double),
        ("alf", ctypes.c_double), ("bet", ctypes.c_double), ("Lchamb", ctypes.c_double),
        ("nxr", ctypes.c_int), ("nyr", ctypes.c_int), ("kg", ctypes.c_int), ("kcm", ctypes.c_int),
        ("a1", ctypes.c_double), ("coord", ctypes.c_int), ("modvis", ctypes.c_int),
        ("beta", ctypes.c_double), ("p0", ctypes.c_double), ("T0", ctypes.c_double),
        ("Twall", ctypes.c_double), ("Rg", ctypes.c_double), ("gamma", ctypes.c_double),
        ("mu", ctypes.c_double), ("kappa", ctypes.c_double), ("itmmax", ctypes.c_int),
        ("itpmax", ctypes.c_int), ("tolm", ctypes.c_double), ("tolt", ctypes.c_double),
        ("solver", ctypes.c_int), ("nitm_u", ctypes.c_int), ("nitm_p", ctypes.c_int),
        ("tol_u", ctypes.c_double), ("tol_p", ctypes.c_double), ("dtmodel", ctypes.c_int),
        ("dt1", ctypes.c_double), ("dt2", ctypes.c_double), ("it1", ctypes.c_int),
        ("it2", ctypes.c_int), ("h0", ctypes.c_double), ("mincc", ctypes.c_double),
        ("maxcc", ctypes.c_double), ("nan_policy", ctypes.c_int), ("ktm", ctypes.c_int),
        ("mix", Mixture), ("modtur", ctypes.c_int), ("prt", ctypes.c_double),
        ("msi_lag", ctypes.c_int),
    ]

    @classmethod
    def from_dict(cls, d):
        """Inverse of as_dict (JSON round trips of float64 values are exact)."""
        c = cls()
        for k, _ in cls._fields_:
            if k != "mix" and k in d:
                setattr(c, k, d[k])
        if d.get("ktm") == 1 and "mix" in d:
            m = d["mix"]
            c.mix.ngs, c.mix.Rg = m["ngs"], m["Rg"]
            for q in range(m["ngs"]):
                c.mix.Xi[q], c.mix.Yi[q], c.mix.Mi[q] = m["Xi"][q], m["Yi"][q], m["Mi"][q]
                c.mix.Ri[q] = m["Ri"][q]
                for k in range(10):
                    c.mix.cpi[q][k] = m["cpi"][q][k]
                for k in range(8):
                    c.mix.mui[q][k] = m["mui"][q][k]
                    c.mix.kpi[q][k] = m["kpi"][q][k]
        return c

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "mix"}
        if self.ktm == 1:
            m = self.mix
            n = m.ngs
            d["mix"] = {"ngs": n, "Rg": m.Rg, "Xi": list(m.Xi)[:n], "Yi": list(m.Yi)[:n],
                        "Mi": list(m.Mi)[:n], "Ri": list(m.Ri)[:n], "cpi": [list(r) for r in m.cpi][:n],
                        "mui": [list(r) for r in m.mui][:n], "kpi": [list(r) for r in m.kpi][:n]}
        return d


class Report(ctypes.Structure):
    """m2d_report: the columns of the residual file (src/mach2d_main.f90:495-516)."""

    _fields_ = [("it", ctypes.c_int), ("dt", ctypes.c_double), ("norm", ctypes.c_double),
                ("normpl", ctypes.c_double), ("rmass", ctypes.c_double), ("fmi", ctypes.c_double),
                ("fme", ctypes.c_double), ("Fd", ctypes.c_double), ("itp_used", ctypes.c_int)]


def euler_cosine_case(nxr=80, nyr=40, **over):
    """Euler, constant properties, C01 cosine nozzle (Lc = 2, Ld = 4, throat
    r = 1 m, inlet r = 2, exit r = 1.8), p0 = 1e6 Pa, T0 = 1000 K, with the
    solver and time-stepper settings of the reference's
    mach2d_input/parametersNozzleEulerPTC.txt deck."""
    c = Case(geom=0, Lc=2.0, Ld=4.0, Rin=2.0, Rout=1.8, nxr=nxr, nyr=nyr, kg=1, kcm=1, a1=5e-6,
             coord=1, modvis=0, beta=0.0, p0=1.0e6, T0=1000.0, Twall=-616.7, Rg=287.0, gamma=1.4,
             mu=1.0e-5, kappa=1.0e-3, itmmax=1, itpmax=20, tolm=1.0e-2, tolt=1.0e-10, solver=0,
             nitm_u=5, nitm_p=20, tol_u=1.0e-2, tol_p=1.0e-2, dtmodel=1, dt1=1e-8, dt2=2e-5,
             it1=100, it2=600, h0=0.01, mincc=0.99, maxcc=0.9999, nan_policy=1)
    for k, v in over.items():
        setattr(c, k, v)
    return c


def n01_case(nxr=20, nyr=10, **over):
    """The reference's own deck: mach2d_input/parametersNozzleEulerPTC.txt with
    geometry_n01.txt (Euler, constant properties, N01 nozzle, 20x10)."""
    c = Case(geom=1, Rth=2.29108e-2, Rin=6.4395244991040e-02, Rout=3.7366383992332e-02,
             Rc1=3.6068e-2, Rc2=4.572e-2, Rc3=4.572e-2, alf=30.0, bet=15.0, Lchamb=2.29108e-2,
             nxr=nxr, nyr=nyr, kg=1, kcm=1, a1=5e-6, coord=1, modvis=0, beta=0.0, p0=1038350.4,
             T0=833.33333333, Twall=-616.7, Rg=287.0, gamma=1.4, mu=1.0e-5, kappa=1.0e-3,
             itmmax=1, itpmax=20, tolm=1.0e-2, tolt=1.0e-10, solver=0, nitm_u=5, nitm_p=20,
             tol_u=1.0e-2, tol_p=1.0e-2, dtmodel=1, dt1=1e-8, dt2=2e-5, it1=100, it2=600,
             h0=0.01, mincc=0.99, maxcc=0.9999, nan_policy=0)
    for k, v in over.items():
        setattr(c, k, v)
    return c


class Simplec:
    """One nozzle instance resident on a GPU."""

    def __init__(self, case, device=0):
        self.case = case
        self._ctx = ctypes.c_void_p()
        L = lib()
        L.m2d_create.argtypes = [ctypes.POINTER(Case), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        check(L.m2d_create(ctypes.byref(case), int(device), ctypes.byref(self._ctx)))
        nx, ny = ctypes.c_int(), ctypes.c_int()
        L.m2d_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        check(L.m2d_dims(self._ctx, ctypes.byref(nx), ctypes.byref(ny)))
        self.nx, self.ny = nx.value, ny.value

    def close(self):
        if self._ctx:
            lib().m2d_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def iterate(self):
        rep = Report()
        L = lib()
        L.m2d_iterate.argtypes = [ctypes.c_void_p, ctypes.POINTER(Report)]
        check(L.m2d_iterate(self._ctx, ctypes.byref(rep)))
        return rep

    def run(self, itmax):
        rep = Report()
        L = lib()
        L.m2d_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Report)]
        check(L.m2d_run(self._ctx, int(itmax), ctypes.byref(rep)))
        return rep

    def run_listing(self, itmax, fh, wlf=1):
        """Like run(), writing the reference's residual listing to `fh`: a row
        every `wlf` iterations and the last one again after the loop
        (src/mach2d_main.f90:420-466)."""
        from .listing import ResidualListing
        lst = ResidualListing(fh, wlf)
        rep = None
        for _ in range(itmax):
            rep = self.iterate()
            lst.write(rep)
            if self.scalar("it_stop") == rep.it:
                break
        if rep is not None:
            lst.write(rep, finished=True)
        return rep

    def main_results(self, rep, rcg=None):
        """write_main_results (mod_intflow_postp.f90:1062-1256) from the device
        fields: (blocks, text).  rcg: the throat's radius of curvature (N01:
        Rc2; C01: that of the diverging cosine, Ld^2 / (0.4 pi^2))."""
        import math
        from .listing import main_results
        c = self.case
        if rcg is None:
            rcg = c.Rc2 if c.geom == 1 else c.Ld ** 2 / (0.4 * math.pi ** 2)
        f = {k: self.field(k) for k in ("x", "y", "re", "ye", "p", "roe", "u", "Uce")}
        nx, ny, y = self.nx, self.ny, f["y"]
        ig = 1
        for i in range(2, nx):
            if y[(ny - 2) * nx + i - 2] < y[(ny - 2) * nx + i - 1]:
                ig = i - 1
                break
        if c.ktm == 0:
            gamma = c.gamma
        else:                                    # gm(T0), as intflow_init takes it
            from .thermo import mixture_eval
            gamma = mixture_eval(c.mix, c.T0)[3]
        return main_results(nx, ny, f["x"], y, f["re"], f["ye"], f["p"], f["roe"], f["u"], f["Uce"],
                            self.scalar("Sg"), rcg, ig, gamma, c.p0, self.scalar("Fpv1D"), self.scalar("Fd1D"),
                            self.scalar("fm1D"), rep.fme)

    def set_msi_schedule(self, variant):
        """m2d_ctx_set_msi_schedule: 0 automatic, 1 one wavefront warp per SM,
        2 two per SM, 3 the one-CTA kernel (same iterates)."""
        L = lib()
        L.m2d_ctx_set_msi_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int]
        check(L.m2d_ctx_set_msi_schedule(self._ctx, int(variant)))

    def set_graph(self, on=True):
        """Run each outer iteration as one captured CUDA graph (m2d_ctx_set_graph)."""
        L = lib()
        L.m2d_ctx_set_graph.argtypes = [ctypes.c_void_p, ctypes.c_int]
        check(L.m2d_ctx_set_graph(self._ctx, 1 if on else 0))

    def set_unet(self, net):
        """Attaches the network solver 3 uses for its p' corrections (None detaches)."""
        L = lib()
        L.m2d_ctx_set_unet.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        check(L.m2d_ctx_set_unet(self._ctx, None if net is None else net._h))
        self._net = net

    def field(self, name):
        n = self._size(name)
        out = np.empty(n, dtype=np.float64)
        L = lib()
        L.m2d_get_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_long]
        check(L.m2d_get_field(self._ctx, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out

    def _fields_call(self, fn, arrays):
        names = list(arrays)
        n = len(names)
        cn = (ctypes.c_char_p * n)(*[k.encode() for k in names])
        ptrs = (ctypes.POINTER(ctypes.c_double) * n)()
        sizes = (ctypes.c_long * n)()
        for k, name in enumerate(names):
            a = arrays[name]
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError("expected C-contiguous float64 arrays")
            ptrs[k] = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            sizes[k] = a.size
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                       ctypes.POINTER(ctypes.POINTER(ctypes.c_double)), ctypes.POINTER(ctypes.c_long)]
        check(fn(self._ctx, n, cn, ptrs, sizes))

    def set_fields(self, arrays):
        """Uploads several named fields {name: float64 array} with one synchronisation."""
        self._fields_call(lib().m2d_set_fields, arrays)

    def get_fields(self, arrays):
        """Downloads several named fields into the given float64 arrays."""
        self._fields_call(lib().m2d_get_fields, arrays)

    def set_field(self, name, values):
        values = np.ascontiguousarray(values, dtype=np.float64)
        L = lib()
        L.m2d_set_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_long]
        check(L.m2d_set_field(self._ctx, name.encode(),
                              values.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), values.size))

    def scalar(self, name):
        v = ctypes.c_double()
        L = lib()
        L.m2d_get_scalar.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        check(L.m2d_get_scalar(self._ctx, name.encode(), ctypes.byref(v)))
        return v.value

    def integrals(self):
        """(fmi, fme, Fd, Cd, p_wall[nx])"""
        vals = [ctypes.c_double() for _ in range(4)]
        pw = np.empty(self.nx, dtype=np.float64)
        L = lib()
        L.m2d_integrals.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_double)] * 5
        check(L.m2d_integrals(self._ctx, *[ctypes.byref(v) for v in vals],
                              pw.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return tuple(v.value for v in vals) + (pw,)

    def _size(self, name):
        N = self.nx * self.ny
        if name in ("au", "av", "at"):
            return 9 * N
        if name == "ap":
            return 5 * N
        if name in ("uin", "vin", "pin", "Tin", "Mw", "plin", "pina", "Tbe", "Tbw"):
            return self.ny
        if name in ("Tbn", "Tbs"):
            return self.nx
        return N


class _BorrowedSimplec(Simplec):
    """A view of one instance of a Batch (the batch owns the context)."""

    def __init__(self, ctx, nx, ny, case):
        self.case = case
        self._ctx = ctx
        self.nx, self.ny = nx, ny

    def close(self):
        self._ctx = ctypes.c_void_p()


class Batch:
    """Many nozzle instances on one GPU (m2d_batch_*): each a full context on
    its own stream, advanced together by `workers` host threads."""

    def __init__(self, cases, device=0, workers=0):
        self.cases = list(cases)
        n = len(self.cases)
        arr = (Case * n)(*self.cases)
        self._b = ctypes.c_void_p()
        L = lib()
        L.m2d_batch_create.argtypes = [ctypes.POINTER(Case), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]
        check(L.m2d_batch_create(arr, n, int(device), int(workers), ctypes.byref(self._b)))
        L.m2d_batch_ctx.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.m2d_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        self.instances = []
        for k in range(n):
            c = ctypes.c_void_p()
            check(L.m2d_batch_ctx(self._b, k, ctypes.byref(c)))
            nx, ny = ctypes.c_int(), ctypes.c_int()
            check(L.m2d_dims(c, ctypes.byref(nx), ctypes.byref(ny)))
            self.instances.append(_BorrowedSimplec(c, nx.value, ny.value, self.cases[k]))

    def __len__(self):
        return len(self.instances)

    def iterate(self, iters=1):
        """Runs `iters` outer iterations of every instance; returns the last
        report of each."""
        n = len(self.instances)
        reps = (Report * n)()
        L = lib()
        L.m2d_batch_iterate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Report)]
        check(L.m2d_batch_iterate(self._b, int(iters), reps))
        return list(reps)

    def set_msi_schedule(self, variant):
        """m2d_batch_set_msi_schedule: the MSI wavefront schedule of every instance."""
        L = lib()
        L.m2d_batch_set_msi_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int]
        check(L.m2d_batch_set_msi_schedule(self._b, int(variant)))

    def autotune(self, iters=2):
        """m2d_batch_autotune: runs the batch's next iterations with each
        candidate MSI schedule and keeps the fastest.  Returns (chosen,
        {schedule: ms per batch iteration})."""
        L = lib()
        L.m2d_batch_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_double)]
        chosen = ctypes.c_int()
        ms = (ctypes.c_double * 4)()
        check(L.m2d_batch_autotune(self._b, int(iters), ctypes.byref(chosen), ms))
        return chosen.value, {v: ms[v] for v in range(4) if ms[v] >= 0}

    def close(self):
        if self._b:
            for s in self.instances:
                s.close()
            lib().m2d_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
