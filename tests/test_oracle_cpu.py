"""Known-answer tests of the CPU oracle (the checker of the GPU tests).

The reference ships no tests or golden vectors and cannot be compiled here,
so the oracle is pinned by analytic results (dense solves, isentropic
relations, exact enthalpy conservation) and by its own committed fixtures.
"""
import json
import math
import os

import numpy as np
import pytest

from _oracle import OracleCase, call
from _systems import dirichlet_system, dense_from_planes, tdma_lines_system
from mach2d_b200.simplec import euler_cosine_case, n01_case

GOLD = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.json")


@pytest.mark.parametrize("nd", [9, 5])
def test_msi_converges_to_dense_solution(nd):
    nx, ny = 12, 9
    a, b = dirichlet_system(nd, nx, ny, seed=3)
    x = np.zeros(nx * ny)
    nit = call(f"msi{nd}_solve", nx, ny, 400, 1e-13, a, b, x)
    ref = np.linalg.solve(dense_from_planes(a, nd, nx, ny), b)
    assert nit < 400
    assert np.max(np.abs(x - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("nd", [9, 5])
def test_tdma_converges_to_dense_solution(nd):
    nx, ny = 10, 7
    a, b = dirichlet_system(nd, nx, ny, seed=5)
    x = np.zeros(nx * ny)
    call(f"tdma2d{nd}", nx, ny, 200, a, b, x)
    ref = np.linalg.solve(dense_from_planes(a, nd, nx, ny), b)
    assert np.max(np.abs(x - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_tdma_line_matches_dense():
    aw, ap, ae, d = tdma_lines_system(n=50, nlines=1, seed=7)
    x = np.zeros(50)
    call("tdma_line", 50, aw[0].copy(), ap[0].copy(), ae[0].copy(), d[0].copy(), x)
    A = np.diag(ap[0]) + np.diag(aw[0, 1:], -1) + np.diag(ae[0, :-1], 1)
    assert np.allclose(x, np.linalg.solve(A, d[0]), rtol=1e-12, atol=1e-12)


def test_msi_single_iteration_reduces_residual():
    nx, ny = 16, 11
    a, b = dirichlet_system(9, nx, ny, seed=11)
    x = np.zeros(nx * ny)
    nit = call("msi9_solve", nx, ny, 1, 1e-30, a, b, x)
    assert nit == 1
    A = dense_from_planes(a, 9, nx, ny)
    assert np.linalg.norm(A @ x - b) < 0.2 * np.linalg.norm(b)


def test_isentropic_relations():
    g, R, p0, T0 = 1.4, 287.0, 1.0e6, 1000.0
    fm = call("get_isentropic_mass_flow", p0, T0, g, R, math.pi)
    # choked mass flow rho* a* A*
    Ts = T0 * 2 / (g + 1)
    ps = p0 * (2 / (g + 1)) ** (g / (g - 1))
    assert fm == pytest.approx(ps / (R * Ts) * math.sqrt(g * R * Ts) * math.pi, rel=1e-13)
    for kf, ar in ((0, 2.5), (1, 2.5), (0, 1.2), (1, 3.9)):
        M = call("get_mach_area", kf, ar, g)
        area = (1 / M) * ((2 / (g + 1)) * (1 + (g - 1) / 2 * M * M)) ** ((g + 1) / (2 * (g - 1)))
        assert area == pytest.approx(ar, rel=1e-10)
        assert (M < 1) == (kf == 0)


def test_gp_ratio_root():
    n, r = 256, 2.1e6
    q = call("get_gp_ratio", n, r)
    assert abs(q ** n + r * (1 - q) - 1) < 1e-6 * r


def test_reference_deck_converges_and_matches_fixture():
    gold = json.load(open(GOLD))["n01_euler_20x10"]
    o = OracleCase(n01_case())
    hist = []
    for _ in range(3000):
        rc, rep = o.iterate()
        assert rc == 0
        if len(hist) < len(gold["history"]):
            hist.append([rep.it, rep.dt, rep.norm, rep.normpl, rep.rmass, rep.fmi, rep.fme, rep.Fd,
                         rep.itp_used])
        if o.scalar("it_stop") == rep.it:
            break
    assert hist == gold["history"]          # the oracle is deterministic
    fin = gold["final"]
    assert rep.it == fin["it"] and rep.normpl < 1e-10
    assert rep.fme / o.scalar("fm1D") == fin["Cd"]
    assert abs(rep.fme / rep.fmi - 1.0) < 1e-10     # mass conserved at convergence


def test_total_enthalpy_is_conserved_for_euler():
    o = OracleCase(euler_cosine_case(20, 10))
    for _ in range(5):
        rc, _ = o.iterate()
        assert rc == 0
    u, v, T = o.field("u"), o.field("v"), o.field("T")
    cp, H = o.scalar("Cpref"), o.scalar("Href")
    nx, ny = o.nx, o.ny
    interior = np.zeros((ny, nx), bool)
    interior[1:-1, 1:-1] = True
    h = cp * T + (u * u + v * v) / 2
    assert np.max(np.abs(h.reshape(ny, nx)[interior] / H - 1)) < 1e-13


def _cartesian_column_case(nx=12, ny=30):
    """Uniform Cartesian grid (unit Jacobian metrics) with a wall at the north."""
    xs = np.arange(nx, dtype=float) * 0.01
    ys = np.arange(ny, dtype=float) * 0.001
    X, Y = np.meshgrid(xs, ys)                       # corners (NE corner of each volume)
    xp, yp = X - 0.005, Y - 0.0005
    f = dict(x=X.reshape(-1).copy(), y=Y.reshape(-1).copy(), xp=xp.reshape(-1).copy(),
             yp=yp.reshape(-1).copy(), xk=np.full(nx * ny, 0.01), yk=np.zeros(nx * ny),
             Jp=np.full(nx * ny, 1.0 / (0.01 * 0.001)), Jn=np.full(nx * ny, 1.0 / (0.01 * 0.001)),
             vln=np.full(nx * ny, 1.8e-5), ro=np.full(nx * ny, 1.2), ron=np.full(nx * ny, 1.2),
             v=np.zeros(nx * ny))
    return nx, ny, f


def test_blomax_oracle_zero_for_uniform_flow_positive_for_shear():
    from _oracle import call as orc
    nx, ny, f = _cartesian_column_case()
    keys = ("x", "y", "xp", "yp", "xk", "yk", "Jp", "Jn", "vln", "ro", "ron", "u", "v")
    f["u"] = np.full(nx * ny, 50.0)
    vt = np.zeros(nx * ny)
    orc("get_eddy_viscosity_blomax", nx, ny, *[f[k] for k in keys], vt, np.zeros(9 * (ny - 2)))
    assert np.all(vt == 0.0)
    d = (f["y"].reshape(ny, nx)[ny - 2:ny - 1, :] - f["yp"].reshape(ny, nx)).clip(0) + 1e-5
    f["u"] = (50.0 * np.tanh(d / 0.005)).reshape(-1).copy()
    orc("get_eddy_viscosity_blomax", nx, ny, *[f[k] for k in keys], vt, np.zeros(9 * (ny - 2)))
    real = vt.reshape(ny, nx)[1:-1, 1:-1]
    assert np.all(real >= 0.0) and np.max(real) > 0.0


def _constant_species_mixture(Rg, gamma, mu, kappa):
    """One species whose cp, mu and k do not depend on T: cp/R = gamma/(gamma-1),
    mu = exp(ln(mu 1e7)) 1e-7, k = exp(ln(k 1e4)) 1e-4."""
    from mach2d_b200.thermo import mixture_init
    Mi = 8.31451 / Rg
    c = gamma / (gamma - 1.0)
    cpi = [c, 0, 0, 0, 0, c, 0, 0, 0, 0]
    lm, lk = math.log(mu * 1e7), math.log(kappa * 1e4)
    return mixture_init(0, [1.0], [Mi], cpi, [0, 0, 0, lm, 0, 0, 0, lm], [0, 0, 0, lk, 0, 0, 0, lk])


def test_mixture_with_constant_species_matches_constant_model():
    """The MIXTURE path of the driver (properties recomputed every iteration,
    src/mach2d_main.f90:112-149) reduces to the CONSTANT one when the species'
    properties do not depend on T: same run to rounding."""
    base = euler_cosine_case(20, 10, modvis=1, Twall=900.0)
    mix = _constant_species_mixture(base.Rg, base.gamma, base.mu, base.kappa)
    var = euler_cosine_case(20, 10, modvis=1, Twall=900.0, ktm=1, mix=mix)
    a, b = OracleCase(base), OracleCase(var)
    assert abs(b.scalar("Cpref") / a.scalar("Cpref") - 1) < 1e-14
    for _ in range(8):
        ra, rb = a.iterate()[1], b.iterate()[1]
        assert ra.itp_used == rb.itp_used
        assert abs(rb.norm / ra.norm - 1) < 1e-9
    for f in ("u", "v", "p", "T"):
        fa, fb = a.field(f), b.field(f)
        assert np.max(np.abs(fa - fb)) <= 1e-9 * np.max(np.abs(fa)), f
    assert np.max(np.abs(b.field("vle")[b.field("vle") != 0] / base.mu - 1)) < 1e-13


def test_mixture_euler_solves_the_energy_equation():
    """ktm = 1 with modvis = 0: T comes from the energy equation (no H
    conservation), cp follows T, and the run stays finite."""
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "air_species.json")))
    from mach2d_b200.thermo import mixture_eval, mixture_init
    mix = mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])
    o = OracleCase(euler_cosine_case(20, 10, ktm=1, mix=mix))
    assert o.scalar("Cpref") == mixture_eval(mix, 1000.0)[0]      # Cpref = cp(T0)
    for _ in range(10):
        rc, rep = o.iterate()
        assert rc == 0 and np.isfinite(rep.norm)
    T, cp = o.field("T"), o.field("cp")
    nx, ny = o.nx, o.ny
    real = np.zeros((ny, nx), bool)
    real[1:-1, 1:-1] = True
    real = real.reshape(-1)
    assert np.std(cp[real]) > 0 and np.all((T[real] > 200) & (T[real] < 1100))


def test_oracle_reproduces_bench_workload_fixture():
    """The first 3 outer iterations of the 512x256 C01 Euler workload are
    bitwise the committed fixture's (tests/golden/make_bench_golden.py)."""
    from mach2d_b200.simplec import Case
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "bench_workloads.json")))
    g = gold["c01_euler_512x256_first20"]
    o = OracleCase(Case.from_dict(g["case"]))
    for row in g["history"][:3]:
        rc, r = o.iterate()
        assert rc == 0
        assert [r.it, r.dt, r.norm, r.normpl, r.rmass, r.fmi, r.fme, r.Fd, r.itp_used] == row
    fin = gold["c01_euler_80x40_converged"]["final"]
    assert fin["it"] == 2 * (fin["it"] // 2) and fin["normpl"] < 1e-10
    assert 1.0 < fin["Cd"] < 1.01


def test_baldwin_lomax_wiring_in_the_oracle_iteration():
    """modtur = 1 adds mu_t (>= 0) to the laminar viscosity at nodes and faces
    and keeps the wall faces laminar; modtur = 0 leaves vtp zero."""
    case = euler_cosine_case(24, 12, modvis=1, Twall=900.0, modtur=1, prt=0.9)
    o = OracleCase(case)
    for _ in range(6):
        rc, _ = o.iterate()
        assert rc == 0
    vtp, vle, vln, vlp = (o.field(f) for f in ("vtp", "vle", "vln", "vlp"))
    nx, ny = o.nx, o.ny
    assert vtp.max() > 0.0 and vtp.min() >= 0.0
    assert np.array_equal(vlp, case.mu + vtp)
    wall = [(ny - 2) * nx + i for i in range(nx)]
    assert np.all(vln[wall] == case.mu)
    assert np.all(vle >= case.mu)
    o2 = OracleCase(euler_cosine_case(24, 12, modvis=1, Twall=900.0))
    o2.iterate()
    assert not o2.field("vtp").any()


def test_extflow_boundary_rows_known_answers():
    """The external-flow oracle's boundary rows, checked by hand on a 6x5
    grid: far-field free-stream value north, slip wall south (Euler), the
    outflow's zero normal gradient east, the axis's zero gradient west, the
    corner averages, interior rows untouched."""
    nx, ny = 6, 5
    N = nx * ny
    xk, yk = np.full(N, 1.0), np.zeros(N)
    u, v = np.full(N, 2.0), np.zeros(N)
    alphae, betae = np.full(N, 1.0), np.zeros(N)
    a, b = np.full(9 * N, 7.0), np.full(N, 7.0)
    call("extflow_set_bcu", nx, ny, 0, 100.0, xk, yk, alphae, betae, u, v, a, b)
    A = a.reshape(9, ny, nx)
    B = b.reshape(ny, nx)
    assert np.all(A[:, 1:-1, 1:-1] == 7.0) and np.all(B[1:-1, 1:-1] == 7.0)
    # north interior: P = 1, b = UF
    assert np.all(A[4, -1, 1:-1] == 1.0) and np.all(B[-1, 1:-1] == 100.0)
    assert np.all(np.delete(A[:, -1, 1:-1], 4, axis=0) == 0.0)
    # south slip: P = N = 1, b = 2 lambda xk = 2 |u| (u along the wall)
    assert np.all(A[4, 0, 1:-1] == 1.0) and np.all(A[7, 0, 1:-1] == 1.0) and np.all(B[0, 1:-1] == 4.0)
    # east: P - W = 0; west with beta = 0: P - E = 0
    assert np.all(A[4, 1:-1, -1] == 1.0) and np.all(A[3, 1:-1, -1] == -1.0)
    assert np.all(A[4, 1:-1, 0] == 1.0) and np.all(A[5, 1:-1, 0] == -1.0)
    # corners: P = 1, three neighbours -1/3
    third = -1.0 / 3.0
    assert (A[4, 0, 0], A[5, 0, 0], A[7, 0, 0], A[8, 0, 0]) == (1.0, third, third, third)
    assert (A[0, -1, -1], A[1, -1, -1], A[3, -1, -1], A[4, -1, -1]) == (third, third, third, 1.0)


def test_extflow_extrapolation_fixed_point_known_answer():
    """The oracle's boundary extrapolation (get_bc_extrapolation_9d) on an
    orthogonal 9x7 grid (beta = 0): after enough sweeps the ring holds the
    far-field density north, copies of the next real cell south, east and
    west, and at each corner the mean of its three neighbours; interior cells
    untouched."""
    nx, ny = 9, 7
    N = nx * ny
    r = np.random.default_rng(5)
    ro0 = r.uniform(1.0, 2.0, N)
    ro = ro0.copy()
    alphae, betae = np.full(N, 1.0), np.zeros(N)
    betan, gamman = np.zeros(N), np.full(N, 1.0)
    call("extflow_extrapolate_ro", nx, ny, 60, 1.225, alphae, betae, betan, gamman, ro)
    R, R0 = ro.reshape(ny, nx), ro0.reshape(ny, nx)
    assert np.array_equal(R[1:-1, 1:-1], R0[1:-1, 1:-1])
    assert np.all(R[-1, 1:-1] == 1.225)
    assert np.allclose(R[0, 1:-1], R[1, 1:-1], rtol=0, atol=1e-14)
    assert np.allclose(R[1:-1, -1], R[1:-1, -2], rtol=0, atol=1e-14)
    assert np.allclose(R[1:-1, 0], R[1:-1, 1], rtol=0, atol=1e-14)
    for (j, i), nb in {(0, 0): [(0, 1), (1, 0), (1, 1)], (0, -1): [(0, -2), (1, -1), (1, -2)],
                       (-1, 0): [(-2, 0), (-2, 1), (-1, 1)], (-1, -1): [(-2, -1), (-2, -2), (-1, -2)]}.items():
        assert abs(R[j, i] - np.mean([R[q] for q in nb])) < 1e-14, (j, i)


def test_extflow_drag_and_T_from_H_known_answers():
    """get_cdfi with a uniform overpressure q on the body: Cdfi = 2 q
    sum(rn yk) / (rb^2 QF); no overpressure, no pressure drag.  T from H with
    a uniform velocity: the static temperature everywhere, ring included."""
    nx, ny = 8, 5
    N = nx * ny
    rn, yk, xk = np.full(N, 0.5), np.full(N, 0.25), np.full(N, 1.0)
    Rg, PF, TF, UF, rb = 287.0, 1.0e5, 250.0, 400.0, 0.5
    QF = PF / (Rg * TF) * UF * UF / 2.0
    z = np.zeros(N)
    for q, want in ((0.0, 0.0), (1000.0, 2.0 * 1000.0 * 5 * 0.125 / (rb * rb * QF))):
        cd = np.zeros(2)
        call("extflow_calc_main_variables", nx, ny, Rg, 0, PF, TF, UF, rb, 6, xk, yk, rn, z, z,
             np.full(N, PF + q), z, z, z, cd)
        assert abs(cd[0] - want) <= 1e-15 * max(1.0, abs(want)) and cd[1] == 0.0
    T = np.zeros(N)
    u, v = np.full(N, 30.0), np.full(N, 40.0)
    tb = [np.zeros(ny), np.zeros(ny), np.zeros(nx), np.zeros(nx)]
    call("extflow_boundary_T_from_H", nx, ny, 1000.0, 3.0e5, u, u, u, v, v, v, T, *tb)
    assert np.all(T == (3.0e5 - 1250.0) / 1000.0)
    assert all(np.all(b[1:-1] == 298.75) for b in tb)
