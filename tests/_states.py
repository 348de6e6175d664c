"""Realistic inputs for routine-level parity: the oracle's own state of a
nozzle after a few outer iterations, optionally perturbed so that every
upwind branch (sign of Uce, Vcn) and the viscous terms are exercised."""
import numpy as np

from _oracle import OracleCase

NAMES = ("x y xp yp xe ye xen yen xk yk xke yke Jp Je Jn alphae gamman betae betan radius re rn rp "
         "fbe fbn p pa T Ta ro roa roe ron g u ua v va ue un ve vn Uce Vcn uea vea una vna cp vlp vle "
         "vln kp ke kn cup sup cvp svp bu bv bt bp pl due dve dun dvn de dn au av at ap "
         "Tbe Tbw Tbn Tbs pin plin Tin uin Mw").split()


def oracle_state(case, iters=3, seed=None, viscous=False):
    o = OracleCase(case)
    for _ in range(iters):
        rc, _ = o.iterate()
        assert rc == 0
    S = {n: o.field(n) for n in NAMES}
    S["nx"], S["ny"] = o.nx, o.ny
    S["dt"] = o.scalar("dt")
    S["Cpref"], S["Href"] = o.scalar("Cpref"), o.scalar("Href")
    S["pina"] = S["pin"] * (1 - 1e-3)
    S["vin"] = np.zeros_like(S["pin"])
    if seed is not None:
        rng = np.random.default_rng(seed)
        N = o.nx * o.ny
        for n in ("Uce", "Vcn", "ue", "ve", "un", "vn"):
            S[n] = S[n] * rng.choice([-1.0, 1.0], N) * rng.uniform(0.5, 1.5, N)
        S["pl"] = rng.standard_normal(N) * 1e2
        S["v"] = S["v"] + rng.standard_normal(N)
    if viscous:
        rng = np.random.default_rng(99)
        N = o.nx * o.ny
        for n in ("vle", "vln", "vlp", "ke", "kn", "kp"):
            S[n] = rng.uniform(1e-5, 2e-5, N)
        S["cp"] = rng.uniform(1000.0, 1100.0, N)
    return S
