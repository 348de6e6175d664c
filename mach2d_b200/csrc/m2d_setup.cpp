// m2d_setup.cpp -- host-side set-up of one nozzle instance: grid, metrics and
// the quasi-1D initial guess.  Runs once per instance, so it stays on the CPU
// (src/mach2d_main.f90:25-84).
//   nozzle contours   N01: src/user/internal_flow/mod_intflow_geometry.f90:29-225
//                     C01: cosine wall, new geometry, inlet at x = 0 (the inlet
//                     boundary conditions measure distances from x = 0,
//                     src/user/internal_flow/mod_intflow.f90:244,907)
//   grids kg = 1, 2   src/grid/mod_grid_procedures.f90:60-279, 349-420
//   metrics, radius   src/grid/mod_grid.f90:237-723
//   initial guess     src/user/internal_flow/mod_intflow.f90:1240-1557
#include "m2d_setup.h"
#include "m2d_thermo.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>

namespace m2d {

namespace {

// integer power as gfortran evaluates x**n (libgcc __powidf2: square and multiply)
double ipow(double x, int m)
{
    unsigned n = m < 0 ? 0u - (unsigned)m : (unsigned)m;
    double y = (n & 1u) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n & 1u) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

struct Grid2 {
    int nx, ny;
    std::vector<double> &x, &y;
    double &at(std::vector<double> &v, int i, int j) { return v[(size_t)(j - 1) * nx + (i - 1)]; }
};

void contour_c01(const m2d_case &c, int nx, int ny, std::vector<double> &x, std::vector<double> &y)
{
    const double pi = std::acos(-1.0);
    const double L = c.Lc + c.Ld;
    for (int i = 1; i <= nx - 1; i++) {
        double xi = ((double)(i - 1) / (double)(nx - 2)) * (L - 0.0) + 0.0;
        double xq = xi - c.Lc;
        double r = (xq <= 0.0) ? 1.0 + 0.5 * (c.Rin - 1.0) * (1.0 - std::cos(pi * xq / c.Lc))
                               : 1.0 + 0.5 * (c.Rout - 1.0) * (1.0 - std::cos(pi * xq / c.Ld));
        x[(size_t)(ny - 2) * nx + i - 1] = xi;
        y[(size_t)(ny - 2) * nx + i - 1] = r;
        x[i - 1] = xi;
        y[i - 1] = 0.0;
    }
}

void contour_n01(const m2d_case &c, int nx, int ny, std::vector<double> &x, std::vector<double> &y)
{
    const double pi = std::acos(-1.0);
    const double alf = c.alf * pi / 180.0, bet = c.bet * pi / 180.0;
    const double x0 = 0.0, y0 = c.Rin, x1 = c.Lchamb, y1 = c.Rin;
    const double x2 = x1 + c.Rc1 * std::sin(alf), y2 = y1 - c.Rc1 * (1.0 - std::cos(alf));
    const double y4 = c.Rth, y3 = y4 + c.Rc2 * (1.0 - std::cos(alf));
    const double x3 = x2 + (y2 - y3) / std::tan(alf);
    const double x4 = x3 + c.Rc2 * std::sin(alf);
    const double x5 = x4 + c.Rc3 * std::sin(bet), y5 = y4 + c.Rc3 * (1.0 - std::cos(bet));
    const double y6 = c.Rout, x6 = x5 + (y6 - y5) / std::tan(bet);
    for (int i = 1; i <= nx - 1; i++) {
        double xv = ((double)(i - 1) / (double)(nx - 2)) * (x6 - x0) + x0, yv;
        if (x0 <= xv && xv <= x1) yv = y0;
        else if (x1 <= xv && xv <= x2) yv = y1 - c.Rc1 + std::sqrt(c.Rc1 * c.Rc1 - (xv - x1) * (xv - x1));
        else if (x2 <= xv && xv <= x3) yv = y2 + (y3 - y2) / (x3 - x2) * (xv - x2);
        else if (x3 <= xv && xv <= x4) yv = y4 + c.Rc2 - std::sqrt(c.Rc2 * c.Rc2 - (xv - x4) * (xv - x4));
        else if (x4 <= xv && xv <= x5) yv = y4 + c.Rc3 - std::sqrt(c.Rc3 * c.Rc3 - (xv - x4) * (xv - x4));
        else if (x5 <= xv && xv <= x6) yv = y5 + (y6 - y5) / (x6 - x5) * (xv - x5);
        else yv = NAN;
        x[(size_t)(ny - 2) * nx + i - 1] = xv;
        y[(size_t)(ny - 2) * nx + i - 1] = yv;
        x[i - 1] = xv;
        y[i - 1] = 0.0;
    }
}

// geometric-progression ratio by bisection, mod_grid_procedures.f90:349-420
double gp_ratio(int n, double r)
{
    double qi, qf, qm = 0.0;
    if (r < n) { qi = 0.1; qf = 1.0 - 1.0e-15; }
    else { qi = 1.0 + 1.0e-15; qf = 10.0; }
    auto fq = [&](double q) { return ipow(q, n) + r * (1.0 - q) - 1.0; };
    for (int it = 1; it <= 1000; it++) {
        qm = 0.5 * qi + 0.5 * qf;
        if (0.0 < fq(qi) * fq(qm)) qi = qm; else qf = qm;
        if (std::fabs(qf - qi) < 1.0e-15) break;
    }
    return qm;
}

void grid_kg(const m2d_case &c, int nx, int ny, std::vector<double> &x, std::vector<double> &y)
{
    for (int i = 1; i <= nx - 1; i++) {
        const double xi = x[i - 1], yi = y[i - 1];
        const size_t top = (size_t)(ny - 2) * nx + i - 1;
        const double xf = x[top], yf = y[top];
        if (c.kg == 1) {
            const double dx = (xf - xi) / (ny - 2), dy = (yf - yi) / (ny - 2);
            for (int j = 2; j <= ny - 2; j++) {
                size_t k = (size_t)(j - 1) * nx + i - 1;
                x[k] = x[k - nx] + dx;
                y[k] = y[k - nx] + dy;
            }
        } else {
            // get_pg_grid with points clustered at the wall (isReversed)
            const int Np = ny - 1;
            const double r = std::sqrt((xf - xi) * (xf - xi) + (yf - yi) * (yf - yi)) / c.a1;
            const double q = gp_ratio(Np - 1, r);
            std::vector<double> t((size_t)Np), d((size_t)Np - 1);
            t[0] = 0.0;
            for (int j = 2; j <= Np - 1; j++) t[j - 1] = t[j - 2] + ipow(q, j - 2) / r;
            t[Np - 1] = 1.0;
            const int n = Np - 1;
            for (int k = 1; k <= n; k++) d[n - k] = t[k] - t[k - 1];
            for (int k = 2; k <= n; k++) t[k - 1] = t[k - 2] + d[k - 2];
            for (int j = 1; j <= ny - 3; j++) {
                size_t k = (size_t)j * nx + i - 1;
                x[k] = xi + (xf - xi) * t[j];
                y[k] = yi + (yf - yi) * t[j];
            }
        }
    }
}

}  // namespace

double mach_area(int kf, double ar, double gamma)
{
    if (std::fabs(ar - 1.0) < 1.0e-15) return 1.0;
    double M0 = kf == 0 ? 1.0e-4 : 1.0, M1 = kf == 0 ? 1.0 : 100.0, M = 1.0;
    auto f = [&](double xx) {
        return std::pow(2.0 * (1.0 + (gamma - 1.0) * (xx * xx) / 2.0) / (gamma + 1.0),
                        (gamma + 1.0) / (gamma - 1.0)) - (xx * ar) * (xx * ar);
    };
    for (int it = 1; it <= 1000; it++) {
        M = 0.5 * (M0 + M1);
        if (f(M) * f(M0) > 0) M0 = M; else M1 = M;
        if (std::fabs(M1 - M0) < 1.0e-15) break;
    }
    return M;
}

int build_instance(const m2d_case &c, HostInstance &h)
{
    const int nx = c.nxr + 2, ny = c.nyr + 2;
    if (c.nxr < 3 || c.nyr < 3) return 2;
    const size_t N = (size_t)nx * ny;
    h.nx = nx; h.ny = ny;
    for (auto &kv : h.planes()) kv.second->assign(N, 0.0);
    auto I = [nx](int i, int j) { return (size_t)(j - 1) * nx + (i - 1); };
    auto &x = h.x, &y = h.y, &xp = h.xp, &yp = h.yp;

    // boundary contour + interior grid (nmf = nmd: the finest grid is the grid)
    if (c.geom == 0) { contour_c01(c, nx, ny, x, y); h.Sg = std::acos(-1.0) * 1.0 * 1.0; }
    else { contour_n01(c, nx, ny, x, y); h.Sg = std::acos(-1.0) * (c.Rth * c.Rth); }
    grid_kg(c, nx, ny, x, y);

    // centroids, mod_grid.f90:237-300
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, j), nps = np - nx, npw = np - 1, npsw = nps - 1;
            if (c.kcm == 1) {
                xp[np] = (x[np] + x[npw] + x[npsw] + x[nps]) / 4.0;
                yp[np] = (y[np] + y[npw] + y[npsw] + y[nps]) / 4.0;
            } else {
                double A1 = 0.5 * (x[npsw] * (y[nps] - y[np]) + x[nps] * (y[np] - y[npsw]) + x[np] * (y[npsw] - y[nps]));
                double A2 = 0.5 * (x[npsw] * (y[np] - y[npw]) + x[np] * (y[npw] - y[npsw]) + x[npw] * (y[npsw] - y[np]));
                xp[np] = ((x[npsw] + x[nps] + x[np]) * A1 + (x[npsw] + x[np] + x[npw]) * A2) / (3.0 * (A1 + A2));
                yp[np] = ((y[npsw] + y[nps] + y[np]) * A1 + (y[npsw] + y[np] + y[npw]) * A2) / (3.0 * (A1 + A2));
            }
        }

    // metrics, mod_grid.f90:304-558
    auto &xe = h.xe, &ye = h.ye, &xen = h.xen, &yen = h.yen, &xk = h.xk, &yk = h.yk;
    auto &xke = h.xke, &yke = h.yke;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
            size_t np = I(i, j), nps = np - nx;
            xe[np] = x[np] - x[nps]; ye[np] = y[np] - y[nps];
            h.alphae[np] = xe[np] * xe[np] + ye[np] * ye[np];
        }
    for (int j = 1; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, j), npw = np - 1;
            xk[np] = x[np] - x[npw]; yk[np] = y[np] - y[npw];
            h.gamman[np] = xk[np] * xk[np] + yk[np] * yk[np];
        }
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 2; i++) {
            size_t np = I(i, j), npe = np + 1;
            xke[np] = xp[npe] - xp[np]; yke[np] = yp[npe] - yp[np];
        }
    for (int j = 2; j <= ny - 1; j++) {
        size_t np = I(2, j), nps = np - nx, npw = np - 1, npsw = nps - 1;
        double fw = (x[npw] + x[npsw]) / 2.0, fe = (x[np] + x[nps]) / 2.0;
        xke[npw] = -3.0 * fw + 4.0 * xp[np] - fe;
        fw = (y[npw] + y[npsw]) / 2.0; fe = (y[np] + y[nps]) / 2.0;
        yke[npw] = -3.0 * fw + 4.0 * yp[np] - fe;
    }
    for (int j = 2; j <= ny - 1; j++) {
        size_t np = I(nx - 1, j), nps = np - nx, npw = np - 1, npsw = nps - 1;
        double fw = (x[npw] + x[npsw]) / 2.0, fe = (x[np] + x[nps]) / 2.0;
        xke[np] = fw - 4.0 * xp[np] + 3.0 * fe;
        fw = (y[npw] + y[npsw]) / 2.0; fe = (y[np] + y[nps]) / 2.0;
        yke[np] = fw - 4.0 * yp[np] + 3.0 * fe;
    }
    for (int j = 2; j <= ny - 2; j++)
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, j), npn = np + nx;
            xen[np] = xp[npn] - xp[np]; yen[np] = yp[npn] - yp[np];
        }
    for (int i = 2; i <= nx - 1; i++) {
        size_t np = I(i, 2), nps = np - nx, npw = np - 1, npsw = nps - 1;
        double fs = (x[nps] + x[npsw]) / 2.0, fn = (x[np] + x[npw]) / 2.0;
        xen[nps] = -3.0 * fs + 4.0 * xp[np] - fn;
        fs = (y[nps] + y[npsw]) / 2.0; fn = (y[np] + y[npw]) / 2.0;
        yen[nps] = -3.0 * fs + 4.0 * yp[np] - fn;
    }
    for (int i = 2; i <= nx - 1; i++) {
        size_t np = I(i, ny - 1), nps = np - nx, npw = np - 1, npsw = nps - 1;
        double fs = (x[nps] + x[npsw]) / 2.0, fn = (x[np] + x[npw]) / 2.0;
        xen[np] = fs - 4.0 * xp[np] + 3.0 * fn;
        fs = (y[nps] + y[npsw]) / 2.0; fn = (y[np] + y[npw]) / 2.0;
        yen[np] = fs - 4.0 * yp[np] + 3.0 * fn;
    }
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
            size_t np = I(i, j);
            h.betae[np] = xke[np] * xe[np] + yke[np] * ye[np];
            h.Je[np] = std::fabs(1.0 / (xke[np] * ye[np] - xe[np] * yke[np]));
        }
    for (int j = 1; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, j);
            h.betan[np] = xk[np] * xen[np] + yk[np] * yen[np];
            h.Jn[np] = std::fabs(1.0 / (xk[np] * yen[np] - xen[np] * yk[np]));
        }
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, j), nps = np - nx, npw = np - 1, npsw = nps - 1;
            double fw = (x[npw] + x[npsw]) / 2.0, fe = (x[np] + x[nps]) / 2.0;
            double fs = (x[nps] + x[npsw]) / 2.0, fn = (x[np] + x[npw]) / 2.0;
            double xkp = fe - fw, xep = fn - fs;
            fw = (y[npw] + y[npsw]) / 2.0; fe = (y[np] + y[nps]) / 2.0;
            fs = (y[nps] + y[npsw]) / 2.0; fn = (y[np] + y[npw]) / 2.0;
            double ykp = fe - fw, yep = fn - fs;
            h.Jp[np] = std::fabs(1.0 / (xkp * yep - xep * ykp));
        }

    // radius, mod_grid.f90:562-723
    auto &re = h.re, &rn = h.rn, &rp = h.rp;
    std::fill(h.radius.begin(), h.radius.end(), 1.0);
    std::fill(re.begin(), re.end(), 1.0);
    std::fill(rn.begin(), rn.end(), 1.0);
    std::fill(rp.begin(), rp.end(), 1.0);
    if (c.coord == 1) {
        h.radius = y;
        for (int i = 1; i <= nx - 1; i++)
            for (int j = 2; j <= ny - 1; j++) { size_t np = I(i, j); re[np] = (y[np] + y[np - nx]) / 2.0; }
        for (int i = 2; i <= nx - 1; i++)
            for (int j = 1; j <= ny - 1; j++) { size_t np = I(i, j); rn[np] = (y[np] + y[np - 1]) / 2.0; }
        rp = yp;
        for (int i = 2; i <= nx - 1; i++) { size_t np = I(i, 1); rp[np] = rn[np] - rp[np + nx] + rn[np]; }
        for (int i = 2; i <= nx - 1; i++) { size_t np = I(i, ny), nps = np - nx; rp[np] = rn[nps] - rp[nps] + rn[nps]; }
        for (int j = 2; j <= ny - 1; j++) { size_t np = I(1, j); rp[np] = re[np] - rp[np + 1] + re[np]; }
        for (int j = 2; j <= ny - 1; j++) { size_t np = I(nx, j), npw = np - 1; rp[np] = re[npw] - rp[npw] + re[npw]; }
        size_t np = I(1, 1);
        rp[np] = 4.0 * y[np] - rp[np + 1] - rp[np + nx] - rp[np + nx + 1];
        np = I(nx, 1);
        rp[np] = 4.0 * y[np - 1] - rp[np - 1] - rp[np + nx] - rp[np + nx - 1];
        np = I(1, ny);
        rp[np] = 4.0 * y[np - nx] - rp[np + 1] - rp[np - nx] - rp[np - nx + 1];
        np = I(nx, ny);
        rp[np] = 4.0 * y[np - nx - 1] - rp[np - 1] - rp[np - nx] - rp[np - nx - 1];
    }

    // boundary-face flags, mach2d_coef.f90:1764-1828
    for (int j = 2; j <= ny - 1; j++) { h.fbe[I(1, j)] = 1.0; h.fbe[I(nx - 1, j)] = 1.0; }
    for (int i = 2; i <= nx - 1; i++) { h.fbn[I(i, ny - 1)] = 1.0; h.fbn[I(i, 1)] = 1.0; }

    // reference values: thermophysical_initialization (mod_thermophysical.f90:20-75)
    // and intflow_init (mod_intflow.f90:72-100); the internal-flow routines take
    // gamma = gm(T0) (:1121, :1186)
    if (c.ktm == 1) {
        h.Rg = c.mix.Rg; h.gamma = m2d::mix_gm(c.mix, c.T0);
        h.Cpref = m2d::mix_cp(c.mix, c.T0);
    } else {
        h.Rg = c.Rg; h.gamma = c.gamma;
        h.Cpref = c.gamma * c.Rg / (c.gamma - 1.0);
    }
    h.Href = h.Cpref * c.T0;

    // quasi-1D isentropic initial guess, mod_intflow.f90:1240-1488
    const double pi = std::acos(-1.0), po = c.p0, T0 = c.T0, gm = h.gamma, Rg = h.Rg, Sg = h.Sg;
    h.fm1D = po * Sg * std::sqrt(gm / (Rg * T0) * std::pow(2.0 / (gm + 1.0), (gm + 1.0) / (gm - 1.0)));
    int ig = 1;
    for (int i = 2; i <= nx - 1; i++)
        if (y[I(i, ny - 1) - 1] < y[I(i, ny - 1)]) { ig = i - 1; break; }
    h.uin.assign(ny, 0.0); h.vin.assign(ny, 0.0); h.pin.assign(ny, 0.0); h.Tin.assign(ny, 0.0);
    h.Mw.assign(ny, 0.0); h.plin.assign(ny, 0.0); h.pina.assign(ny, 0.0);
    h.M1D.assign(nx, 0.0); h.p1D.assign(nx, 0.0); h.T1D.assign(nx, 0.0); h.u1D.assign(nx, 0.0);
    auto &p = h.p, &T = h.T, &u = h.u, &v = h.v;
    for (int i = 2; i <= nx - 1; i++) {
        size_t np = I(i, ny - 1);
        double Si = pi * (rn[np] * rn[np]);
        int kf = i > ig ? 1 : 0;
        h.M1D[i - 1] = mach_area(kf, Si / Sg, gm);
        double aux = 1.0 + 0.5 * (gm - 1.0) * (h.M1D[i - 1] * h.M1D[i - 1]);
        h.p1D[i - 1] = po * std::pow(aux, -gm / (gm - 1.0));
        h.T1D[i - 1] = T0 / aux;
        h.u1D[i - 1] = h.M1D[i - 1] * std::sqrt(gm * Rg * h.T1D[i - 1]);
        for (int j = 1; j <= ny; j++) {
            np = I(i, j);
            p[np] = h.p1D[i - 1]; T[np] = h.T1D[i - 1]; u[np] = h.u1D[i - 1];
            if (j > 1 && j < ny - 1) { h.un[np] = h.u1D[i - 1]; h.Vcn[np] = -h.un[np] * yk[np]; }
        }
    }
    // intflow_extrapolate_u_v_to_fictitious on the initial field (modvis aware)
    {
        for (int j = 2; j <= ny - 1; j++) {
            size_t np = I(1, j), npe = np + 1, npee = np + 2;
            u[np] = u[npe] + 2.0 * xp[npe] / (xp[npee] - xp[npe]) * (u[npe] - u[npee]);
            v[np] = -v[npe];
        }
        for (int j = 2; j <= ny - 1; j++) {
            size_t np = I(nx, j), npw = np - 1, npww = np - 2;
            u[np] = u[npw] + 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]) * (u[npw] - u[npww]);
            v[np] = v[npw] + 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]) * (v[npw] - v[npww]);
        }
        for (int i = 1; i <= nx; i++) { size_t np = I(i, 1); u[np] = u[np + nx]; v[np] = -v[np + nx]; }
        std::vector<double> ubn(nx, 0.0), vbn(nx, 0.0);
        if (c.modvis != 1) north_slip_host(nx, ny, x, xp, xk, yk, u, v, ubn, vbn);
        for (int i = 1; i <= nx; i++) {
            size_t np = I(i, ny), nps = np - nx;
            if (c.modvis == 1) { u[np] = -u[nps]; v[np] = -v[nps]; }
            else { u[np] = -u[nps] + 2.0 * ubn[i - 1]; v[np] = -v[nps] + 2.0 * vbn[i - 1]; }
        }
    }
    for (int j = 2; j <= ny - 1; j++) {
        size_t np = I(1, j), npe = np + 1;
        h.uin[j - 1] = (u[np] + u[npe]) / 2.0;
        h.vin[j - 1] = 0.0;
        h.Tin[j - 1] = T0 - (gm - 1.0) / (2.0 * gm * Rg) * (h.uin[j - 1] * h.uin[j - 1] + h.vin[j - 1] * h.vin[j - 1]);
        h.Mw[j - 1] = std::sqrt((h.uin[j - 1] * h.uin[j - 1] + h.vin[j - 1] * h.vin[j - 1]) / (gm * Rg * h.Tin[j - 1]));
        h.pin[j - 1] = po * std::pow(1.0 + 0.5 * (gm - 1.0) * (h.Mw[j - 1] * h.Mw[j - 1]), -gm / (gm - 1.0));
    }
    for (int j = 2; j <= ny - 1; j++) {
        size_t np = I(1, j), npe = np + 1;
        p[np] = 2.0 * h.pin[j - 1] - p[npe];
        T[np] = 2.0 * h.Tin[j - 1] - T[npe];
    }
    for (int j = 2; j <= ny - 1; j++) {
        size_t np = I(nx, j), npw = np - 1, npww = np - 2;
        double fac = 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]);
        p[np] = p[npw] + fac * (p[npw] - p[npww]);
        T[np] = T[npw] + fac * (T[npw] - T[npww]);
    }
    const size_t cor[4][2] = {{I(1, 1), I(1, 2)}, {I(nx, 1), I(nx, 2)}, {I(1, ny), I(1, ny - 1)}, {I(nx, ny), I(nx, ny - 1)}};
    for (auto &cc : cor) { p[cc[0]] = p[cc[1]]; T[cc[0]] = T[cc[1]]; }
    for (int i = 1; i <= nx - 1; i++) {
        size_t np = I(i, ny - 1);
        double Si = pi * (h.radius[np] * h.radius[np]);
        int kf = i > ig ? 1 : 0;
        double Me = mach_area(kf, Si / Sg, gm);
        double aux = 1.0 + 0.5 * (gm - 1.0) * (Me * Me);
        double pe = po * std::pow(aux, -gm / (gm - 1.0));
        double Te = T0 / aux;
        double ue1 = Me * std::sqrt(gm * Rg * Te);
        for (int j = 2; j <= ny - 1; j++) { np = I(i, j); h.ue[np] = ue1; h.Uce[np] = ue1 * ye[np]; }
        if (i == 1) { h.u1D[0] = ue1; h.p1D[0] = pe; h.T1D[0] = Te; h.M1D[0] = Me; }
        if (i == nx - 1) {
            h.u1D[nx - 1] = ue1; h.p1D[nx - 1] = pe; h.T1D[nx - 1] = Te; h.M1D[nx - 1] = Me;
            h.Fd1D = h.fm1D * ue1;
            h.Fpv1D = pe * Si;
        }
    }
    // velocities at boundary faces
    {
        for (int j = 2; j <= ny - 1; j++) {
            size_t np = I(1, j), npe = np + 1;
            h.ue[np] = (u[np] + u[npe]) / 2.0; h.ve[np] = 0.0;
            h.Uce[np] = h.ue[np] * ye[np] - h.ve[np] * xe[np];
        }
        for (int j = 2; j <= ny - 1; j++) {
            size_t np = I(nx - 1, j), npe = np + 1;
            h.ue[np] = (u[np] + u[npe]) / 2.0; h.ve[np] = (v[np] + v[npe]) / 2.0;
            h.Uce[np] = h.ue[np] * ye[np] - h.ve[np] * xe[np];
        }
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, 1), npn = np + nx;
            h.un[np] = (u[np] + u[npn]) / 2.0; h.vn[np] = 0.0; h.Vcn[np] = 0.0;
        }
        std::vector<double> ubn(nx, 0.0), vbn(nx, 0.0);
        if (c.modvis == 0) north_slip_host(nx, ny, x, xp, xk, yk, u, v, ubn, vbn);
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, ny - 1);
            h.un[np] = ubn[i - 1]; h.vn[np] = vbn[i - 1]; h.Vcn[np] = 0.0;
        }
    }
    // densities
    for (size_t k = 0; k < N; k++) h.ro[k] = p[k] / (Rg * T[k]);
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
            size_t np = I(i, j), npe = np + 1;
            double ae = std::copysign(0.5, h.Uce[np]);
            h.roe[np] = (0.5 + ae) * h.ro[np] + (0.5 - ae) * h.ro[npe] + c.beta * ae * (h.ro[npe] - h.ro[np]);
        }
    for (int j = 1; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            size_t np = I(i, j), npn = np + nx;
            double an = std::copysign(0.5, h.Vcn[np]);
            h.ron[np] = (0.5 + an) * h.ro[np] + (0.5 - an) * h.ro[npn] + c.beta * an * (h.ro[npn] - h.ro[np]);
        }
    h.Tbw = h.Tin;
    h.Tbs = h.T1D;
    h.Tbn = h.T1D;
    h.Tbe.assign(ny, h.T1D[nx - 2]);
    // constant properties (get_cp_mu_kappa_initialization); the MIXTURE model's
    // fields are computed on the device by m2d_create from T and Tbn..Tbw
    if (c.ktm != 1) std::fill(h.cp.begin(), h.cp.end(), h.Cpref);
    if (c.modvis == 1 && c.ktm != 1) {
        std::fill(h.vlp.begin(), h.vlp.end(), c.mu); std::fill(h.vle.begin(), h.vle.end(), c.mu);
        std::fill(h.vln.begin(), h.vln.end(), c.mu); std::fill(h.kp.begin(), h.kp.end(), c.kappa);
        std::fill(h.ke.begin(), h.ke.end(), c.kappa); std::fill(h.kn.begin(), h.kn.end(), c.kappa);
    }
    // first time step (tstepper_dt0)
    if (c.dtmodel == 1) {
        double dt = 1.0e10;
        for (int i = 2; i <= nx - 1; i++)
            for (int j = 2; j <= ny - 1; j++) {
                size_t np = I(i, j);
                double aux = 1.0 / std::sqrt(h.Jp[np] * (u[np] * u[np] + v[np] * v[np]));
                if (dt > aux) dt = aux;
            }
        h.dt0 = dt * 0.25;
    } else {
        h.dt0 = ramp_dt(0, c);
    }
    return 0;
}

double ramp_dt(int it, const m2d_case &c)
{
    double dt = 0.0;
    if (it + 1 <= c.it1) dt = c.dt1;
    if (it + 1 > c.it1 && it + 1 < c.it2) dt = c.dt1 + (c.dt2 - c.dt1) * (double)(it + 1 - c.it1) / (double)(c.it2 - c.it1);
    if (it + 1 >= c.it2) dt = c.dt2;
    return dt;
}

void north_slip_host(int nx, int ny, const std::vector<double> &x, const std::vector<double> &xp,
                     const std::vector<double> &xk, const std::vector<double> &yk,
                     const std::vector<double> &u, const std::vector<double> &v,
                     std::vector<double> &ubn, std::vector<double> &vbn)
{
    const int j = ny - 1;
    for (int i = 2; i <= nx - 1; i++) {
        size_t np = (size_t)(j - 1) * nx + i - 1;
        double Up = std::sqrt(u[np] * u[np] + v[np] * v[np]);
        double sg = std::copysign(1.0, xk[np] * u[np] + yk[np] * v[np]);
        double t = std::sqrt(xk[np] * xk[np] + yk[np] * yk[np]);
        ubn[i - 1] = sg * Up * (xk[np] / t);
        vbn[i - 1] = sg * Up * (yk[np] / t);
    }
    size_t np = (size_t)(j - 1) * nx, npe = np + 1, npee = npe + 1;
    ubn[0] = ubn[1] + (ubn[1] - ubn[2]) * (xp[npe] - x[np]) / (xp[npee] - xp[npe]);
    vbn[0] = vbn[1] + (vbn[1] - vbn[2]) * (xp[npe] - x[np]) / (xp[npee] - xp[npe]);
    np = (size_t)(j - 1) * nx + nx - 1;
    size_t npw = np - 1, npww = npw - 1;
    ubn[nx - 1] = ubn[nx - 2] + (ubn[nx - 2] - ubn[nx - 3]) * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]);
    vbn[nx - 1] = vbn[nx - 2] + (vbn[nx - 2] - vbn[nx - 3]) * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]);
}

}  // namespace m2d
