"""Output files of the reference, written from the device-resident iteration:
the residual listing of src/mach2d_main.f90:473-520 (calc_print_main_variables
with intflow_calc_main_variables, src/user/internal_flow/mod_intflow.f90:1647-1666)
and the main-results report of write_main_results
(src/user/internal_flow/mod_intflow_postp.f90:1062-1256), in the same
Fortran edit descriptors, so that files from both programs diff line by line.
"""
import math

PR = 1.013e5   # atmospheric pressure at sea level (mod_intflow_postp.f90:58)
GO = 9.81      # gravitational acceleration (mod_intflow_postp.f90:59)


def fortran_a(s, w):
    """Aw output: right-justified in w columns, the leftmost w characters if longer."""
    s = str(s)
    return s[:w] if len(s) >= w else " " * (w - len(s)) + s


def fortran_i(v, w):
    s = str(int(v))
    return "*" * w if len(s) > w else fortran_a(s, w)


def fortran_es(x, w, d):
    """ESw.d (and 1PEw.d): one digit before the point, d after, exponent
    E+dd, or +ddd without the E when its magnitude exceeds 99."""
    if math.isnan(x):
        return fortran_a("NaN", w)
    if math.isinf(x):
        return fortran_a("-Infinity" if x < 0 else "Infinity", w)
    if x == 0.0:
        mant, exp = "0." + "0" * d, 0
        sign = "-" if math.copysign(1.0, x) < 0 else ""
    else:
        sign = "-" if x < 0 else ""
        s = f"{abs(x):.{d}e}"              # round-half-even on the decimal expansion of the double
        m, e = s.split("e")
        mant, exp = m, int(e)
    if abs(exp) <= 99:
        es = f"E{'+' if exp >= 0 else '-'}{abs(exp):02d}"
    else:
        es = f"{'+' if exp >= 0 else '-'}{abs(exp):03d}"
    out = sign + mant + es
    return "*" * w if len(out) > w else fortran_a(out, w)


class ResidualListing:
    """The residual file: a header at it = 1, then a row every `wlf`
    iterations and at the end (format (I10, 4(1X,ES14.7), A) plus the
    internal-flow message 3(1X,ES23.16) of fmi, fme/fmi, Fd)."""

    def __init__(self, fh, wlf=1):
        self.fh, self.wlf = fh, wlf

    @staticmethod
    def header():
        msg1 = "".join(" " + fortran_a(s, 23) for s in ("fmi", "fme/fmi", "Fd"))
        return fortran_a("it", 10) + "".join(" " + fortran_a(s, 14) for s in
                                             ("dt", "norm", "max(|pl|)/p_avg", "rmass")) + msg1

    @staticmethod
    def row(rep):
        msg2 = "".join(" " + fortran_es(v, 23, 16) for v in (rep.fmi, rep.fme / rep.fmi, rep.Fd))
        return fortran_i(rep.it, 10) + "".join(" " + fortran_es(v, 14, 7) for v in
                                               (rep.dt, rep.norm, rep.normpl, rep.rmass)) + msg2

    def write(self, rep, finished=False):
        if rep.it == 1:
            self.fh.write(self.header() + "\n")
        if rep.it % self.wlf == 0 or finished:
            self.fh.write(self.row(rep) + "\n")


def main_results(nx, ny, x, y, re, ye, p, roe, u, Uce, Sg, rcg, ig, gamma, po, Fpv1D, Fd1D, fm1D, fme):
    """The values of write_main_results (mod_intflow_postp.f90:1062-1256) as a
    dict of lists [(value, label)] per block, and its text.  ig: the throat
    column (1-based) of write_nozzle_parameters (:814-860)."""
    pi = math.acos(-1.0)
    I = lambda i, j: (j - 1) * nx + i - 1   # noqa: E731
    Sex = pi * (y[I(nx - 1, ny - 1)] ** 2)
    Fp1D = Fpv1D - PR * Sex
    F1D = Fd1D + Fp1D
    Fv1D = Fd1D + Fpv1D
    Fo = po * Sg
    CF1D, CFv1D = F1D / Fo, Fv1D / Fo
    ce1D, c1D, cv1D = Fo / fm1D, F1D / fm1D, Fv1D / fm1D
    Is1D, Isv1D = c1D / GO, cv1D / GO
    rcag = rcg / y[I(ig, ny - 1)]
    KL1 = (gamma + 1) / ((1 + rcag) ** 2)
    KL2 = (8 * gamma - 27) / (2304 * (1 + rcag))
    KL3 = 754 * (gamma ** 2) - (757 * gamma) + 3633
    KL4 = 276480 * ((1 + rcag) ** 2)
    CdKL = 1 - KL1 * ((1 / 9.6e+1) - KL2 + (KL3 / KL4))
    Fd = Fp = Fpv = 0.0
    i = nx - 1
    for j in range(2, ny):
        np_, npe = I(i, j), I(i, j) + 1
        Fd = Fd + re[np_] * roe[np_] * Uce[np_] * u[npe]
        Fp = Fp + (p[npe] - PR) * re[np_] * ye[np_]
        Fpv = Fpv + p[npe] * re[np_] * ye[np_]
    Fd, Fp, Fpv = Fd * 2 * pi, Fp * 2 * pi, Fpv * 2 * pi
    F, Fv = Fd + Fp, Fd + Fpv
    CF, CFv = F / Fo, Fv / Fo
    ce, c, cv = Fo / fme, F / fme, Fv / fme
    Is, Isv = c / GO, cv / GO
    q1d = [(fm1D, "fm1D:  mass flow rate (kg/s)"), (Fd1D, "Fd1D:  dynamic thrust (N)"),
           (Fp1D, "Fp1D:  dynamic thrust at sea level (p = 101325 Pa) (N)"),
           (Fpv1D, "Fpv1D: thrust of pressure in the vacuum (N)"), (F1D, "F1D:   total thrust at sea level (N)"),
           (Fv1D, "Fv1D:  total thrust in the vacuum (N)"), (Fo, "Fo:    standard thrust (N)"),
           (CF1D, "CF1D:  thrust coefficient at sea level (dimensionless)"),
           (CFv1D, "CFv1D: thrust coefficient in the vacuum (dimensionless)"),
           (ce1D, "ce1D:  characteristic velocity (m/s)"),
           (c1D, "c1D:   velocity of efective ejection at the sea level (m/s)"),
           (cv1D, "cv1D:  velocity of efective ejection in the vacuum (m/s)"),
           (Is1D, "Is1D:  specific impulse at sea level (s)"), (Isv1D, "Isv1D: specific impulse in the vacuum (s)")]
    num = [(fme, "fme: mass flow rate (kg/s)"), (Fd, "Fd:  dynamic thrust (N)"),
           (Fp, "Fp:  thrust of pressure at sea level (p = 101325 Pa) (N)"),
           (Fpv, "Fpv: thrust of pressure in the vacuum (N)"), (F, "F:   total thrust at sea level (N)"),
           (Fv, "Fv:  total thrust in the vacuum (N)"), (Fo, "Fo:  standard thrust (N)"),
           (CF, "CF:  thrust coefficient at sea level (dimensionless)"),
           (CFv, "CFv: thrust coefficient in the vacuum (dimensionless)"),
           (ce, "ce:  characteristic velocity (m/s)"), (c, "c:   velocity of efective ejection at sea level (m/s)"),
           (cv, "cv:  velocity of efective ejection in the vacuum (m/s)"),
           (Is, "Is:  specific impulse at sea level (s)"), (Isv, "Isv: specific impulse in the vacuum (s)")]
    eff = [(fme / fm1D, "discharge coefficient"), (Fd / Fd1D, "dynamic thrust"),
           (Fp / Fp1D, "pressure thrust at sea level (p = 101325 Pa)"), (Fpv / Fpv1D, "pressure thrust in the vacuum"),
           (F / F1D, "total thrust at sea level"), (Fv / Fv1D, "total thrust in the vacuum"),
           (CF / CF1D, "thrust coefficient at sea level"), (CFv / CFv1D, "thrust coefficient in the vacuum"),
           (ce / ce1D, "characterist velocity"), (c / c1D, "velocity of efective ejection at sea level"),
           (cv / cv1D, "velocity of efective ejection in the vacuum"), (Is / Is1D, "specific impulse at sea level"),
           (Isv / Isv1D, "specific impulse at vacuum")]
    blocks = {"q1d": q1d, "kl": [(CdKL, "CdKL: discharge coefficient of Kliegel and Levine (dimensionless)")],
              "numeric": num, "efficiency": eff}
    lines = ["", " *** Analytic solution of the Q1D isentropic flow ***", ""]
    lines += [fortran_es(v, 25, 15) + " = " + t for v, t in q1d]
    lines += ["", " *** Analytic solution 2D ***", ""]
    lines += [fortran_es(CdKL, 25, 15) + " = " + blocks["kl"][0][1]]
    lines += ["", " *** Numeric solution 2D ***", ""]
    lines += [fortran_es(v, 25, 15) + " = " + t for v, t in num]
    lines += ["", " *** Efficiency: numerical solution 2D / analytic Q1D (dimensionless) ***", ""]
    lines += [fortran_es(v, 25, 15) + " = " + t for v, t in eff]
    return blocks, "\n".join(lines) + "\n"
