// m2d_setup.cpp -- host-side part of the set-up of one nozzle instance
// (src/mach2d_main.f90:25-84): the grid nodes and the O(nx + ny) quasi-1D
// strips of the initial guess, the parts that call cos, pow and the Mach-area
// bisection, so that they round as the reference's x86-64 build does.  The
// metrics and every O(nx ny) part of the initial guess are computed on the
// device from the uploaded nodes (m2d_grid.cu, m2d_create).
//   nozzle contours   N01: src/user/internal_flow/mod_intflow_geometry.f90:29-225
//                     C01: cosine wall, new geometry, inlet at x = 0 (the inlet
//                     boundary conditions measure distances from x = 0,
//                     src/user/internal_flow/mod_intflow.f90:244,907)
//   grids kg = 1, 2   src/grid/mod_grid_procedures.f90:60-279, 349-420
//   initial guess     src/user/internal_flow/mod_intflow.f90:1240-1557 (the
//                     strips; the rest in m2d_grid.cu)
#include "m2d_setup.h"
#include "m2d_grid.cuh"
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
    h.x.assign(N, 0.0); h.y.assign(N, 0.0);
    auto I = [nx](int i, int j) { return (size_t)(j - 1) * nx + (i - 1); };
    const std::vector<double> &y = h.y;

    // boundary contour + interior grid (nmf = nmd: the finest grid is the grid)
    if (c.geom == 0) { contour_c01(c, nx, ny, h.x, h.y); h.Sg = std::acos(-1.0) * 1.0 * 1.0; }
    else { contour_n01(c, nx, ny, h.x, h.y); h.Sg = std::acos(-1.0) * (c.Rth * c.Rth); }
    grid_kg(c, nx, ny, h.x, h.y);

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

    // quasi-1D isentropic strips of the initial guess (mod_intflow.f90:1303-1349,
    // 1423-1472): the face radii of the north row come from the same
    // expressions the device's get_radius uses
    const double pi = std::acos(-1.0), po = c.p0, T0 = c.T0, gm = h.gamma, Rg = h.Rg, Sg = h.Sg;
    h.fm1D = po * Sg * std::sqrt(gm / (Rg * T0) * std::pow(2.0 / (gm + 1.0), (gm + 1.0) / (gm - 1.0)));
    int ig = 1;
    for (int i = 2; i <= nx - 1; i++)
        if (y[I(i, ny - 1) - 1] < y[I(i, ny - 1)]) { ig = i - 1; break; }
    h.M1D.assign(nx, 0.0); h.p1D.assign(nx, 0.0); h.T1D.assign(nx, 0.0); h.u1D.assign(nx, 0.0);
    h.ue1D.assign(nx, 0.0);
    for (int i = 2; i <= nx - 1; i++) {
        const double rn = rn_value(c.coord, nx, ny, y.data(), i, ny - 1);
        const double Si = pi * (rn * rn);
        const int kf = i > ig ? 1 : 0;
        h.M1D[i - 1] = mach_area(kf, Si / Sg, gm);
        const double aux = 1.0 + 0.5 * (gm - 1.0) * (h.M1D[i - 1] * h.M1D[i - 1]);
        h.p1D[i - 1] = po * std::pow(aux, -gm / (gm - 1.0));
        h.T1D[i - 1] = T0 / aux;
        h.u1D[i - 1] = h.M1D[i - 1] * std::sqrt(gm * Rg * h.T1D[i - 1]);
    }
    h.col.assign(4 * (size_t)nx, 0.0);
    std::copy(h.p1D.begin(), h.p1D.end(), h.col.begin());
    std::copy(h.T1D.begin(), h.T1D.end(), h.col.begin() + nx);
    std::copy(h.u1D.begin(), h.u1D.end(), h.col.begin() + 2 * nx);
    for (int i = 1; i <= nx - 1; i++) {
        const double r = radius_value(c.coord, nx, y.data(), i, ny - 1);
        const double Si = pi * (r * r);
        const int kf = i > ig ? 1 : 0;
        const double Me = mach_area(kf, Si / Sg, gm);
        const double aux = 1.0 + 0.5 * (gm - 1.0) * (Me * Me);
        const double pe = po * std::pow(aux, -gm / (gm - 1.0));
        const double Te = T0 / aux;
        const double ue1 = Me * std::sqrt(gm * Rg * Te);
        h.ue1D[i - 1] = ue1;
        if (i == 1) { h.u1D[0] = ue1; h.p1D[0] = pe; h.T1D[0] = Te; h.M1D[0] = Me; }
        if (i == nx - 1) {
            h.u1D[nx - 1] = ue1; h.p1D[nx - 1] = pe; h.T1D[nx - 1] = Te; h.M1D[nx - 1] = Me;
            h.Fd1D = h.fm1D * ue1;
            h.Fpv1D = pe * Si;
        }
    }
    std::copy(h.ue1D.begin(), h.ue1D.end(), h.col.begin() + 3 * nx);
    h.Tbs = h.T1D;
    h.Tbn = h.T1D;
    h.Tbe.assign(ny, h.T1D[nx - 2]);
    h.dt0 = ramp_dt(0, c);      // replaced by the device's dt0 when dtmodel = 1
    return 0;
}

void inlet_strips(const m2d_case &c, HostInstance &h, const std::vector<double> &uin)
{
    const int ny = h.ny;
    const double po = c.p0, T0 = c.T0, gm = h.gamma, Rg = h.Rg;
    h.uin = uin;
    h.vin.assign(ny, 0.0); h.pin.assign(ny, 0.0); h.Tin.assign(ny, 0.0); h.Mw.assign(ny, 0.0);
    for (int j = 2; j <= ny - 1; j++) {
        const double u = h.uin[j - 1], v = h.vin[j - 1];
        h.Tin[j - 1] = T0 - (gm - 1.0) / (2.0 * gm * Rg) * (u * u + v * v);
        h.Mw[j - 1] = std::sqrt((u * u + v * v) / (gm * Rg * h.Tin[j - 1]));
        h.pin[j - 1] = po * std::pow(1.0 + 0.5 * (gm - 1.0) * (h.Mw[j - 1] * h.Mw[j - 1]), -gm / (gm - 1.0));
    }
    h.Tbw = h.Tin;
}

double ramp_dt(int it, const m2d_case &c)
{
    double dt = 0.0;
    if (it + 1 <= c.it1) dt = c.dt1;
    if (it + 1 > c.it1 && it + 1 < c.it2) dt = c.dt1 + (c.dt2 - c.dt1) * (double)(it + 1 - c.it1) / (double)(c.it2 - c.it1);
    if (it + 1 >= c.it2) dt = c.dt2;
    return dt;
}

}  // namespace m2d
