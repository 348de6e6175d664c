/*
 * thermo.c -- gas-mixture thermophysical model
 * (src/thermophysical/mod_class_thermophysical_mixture.f90), the field
 * routines of src/thermophysical/mod_thermophysical.f90 and the boundary
 * averages of src/util/mod_field_operations.f90.
 * TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).
 *
 * Constant integer powers follow gfortran -O2's expansion: T**2 = T*T,
 * T**3 = (T*T)*T, T**4 = (T*T)*(T*T).
 */
#include <math.h>
#include <string.h>
#include "m2d_oracle.h"

#define IDX(i, j) ((long)nx * ((j) - 1) + (i) - 1)

int orc_mixture_init(int base, int ngs, const double *fr, const double *Mi, const double *cpi,
                     const double *mui, const double *kpi, orc_mixture *out)
{   /* init, mod_class_thermophysical_mixture.f90:56-224 */
    orc_mixture m;
    memset(&m, 0, sizeof m);
    const double Ru = 8.31451000e+00;
    for (int k = 0; k < ngs; k++) {
        if (!(fr[k] > 1.0e-8)) continue;
        if (m.ngs == ORC_MAX_SPECIES) return 2;
        const int q = m.ngs++;
        if (base == 0) m.Xi[q] = fr[k]; else m.Yi[q] = fr[k];
        m.Mi[q] = Mi[k];
        for (int c = 0; c < 10; c++) m.cpi[q][c] = cpi[10 * k + c];
        for (int c = 0; c < 8; c++) m.mui[q][c] = mui[8 * k + c];
        for (int c = 0; c < 8; c++) m.kpi[q][c] = kpi[8 * k + c];
    }
    if (m.ngs == 0) return 2;
    double s = 0.0;
    for (int q = 0; q < m.ngs; q++) s += (base == 0) ? m.Xi[q] : m.Yi[q];
    if (fabs(1.0 - s) > 2.220446049250313e-16 * 10.0) return 2;
    double Mg = 0.0;
    if (base == 0) {
        for (int q = 0; q < m.ngs; q++) Mg += m.Xi[q] * m.Mi[q];
        for (int q = 0; q < m.ngs; q++) m.Yi[q] = m.Xi[q] * m.Mi[q] / Mg;
    } else {
        double den = 0.0;
        for (int q = 0; q < m.ngs; q++) den += m.Yi[q] / m.Mi[q];
        for (int q = 0; q < m.ngs; q++) m.Xi[q] = (m.Yi[q] / m.Mi[q]) / den;
        for (int q = 0; q < m.ngs; q++) Mg += m.Xi[q] * m.Mi[q];
    }
    for (int q = 0; q < m.ngs; q++) m.Ri[q] = Ru / m.Mi[q];
    m.Rg = Ru / Mg;
    *out = m;
    return 0;
}

static double cp_i(double T, double Ri, const double *a)
{   /* :563-581 */
    double v;
    if (T <= 1000.0) v = a[0] + a[1] * T + a[2] * (T * T) + a[3] * (T * T * T) + a[4] * ((T * T) * (T * T));
    else v = a[5] + a[6] * T + a[7] * (T * T) + a[8] * (T * T * T) + a[9] * ((T * T) * (T * T));
    return v * Ri;
}
static double transport_i(double T, const double *a, double scale)
{   /* mu_i :639-654 (1e-7), kp_i :712-727 (1e-4) */
    if (T <= 1000.0) return exp(a[0] * log(T) + a[1] / T + a[2] / (T * T) + a[3]) * scale;
    return exp(a[4] * log(T) + a[5] / T + a[6] / (T * T) + a[7]) * scale;
}
double orc_mix_cp(const orc_mixture *m, double T)
{   /* cp_mix :539-559 */
    double s = 0.0;
    for (int i = 0; i < m->ngs; i++) s = s + m->Yi[i] * cp_i(T, m->Ri[i], m->cpi[i]);
    return s;
}
static double wilke(const orc_mixture *m, double T, int visc)
{   /* mu_mix :585-635, kp_mix :658-708 */
    double r[ORC_MAX_SPECIES];
    for (int i = 0; i < m->ngs; i++) r[i] = visc ? transport_i(T, m->mui[i], 1.0e-7) : transport_i(T, m->kpi[i], 1.0e-4);
    double s = 0.0;
    for (int i = 0; i < m->ngs; i++) {
        double d = 0.0;
        for (int j = 0; j < m->ngs; j++) {
            double t = 1.0 + sqrt(r[i] / r[j] * sqrt(m->Mi[j] / m->Mi[i]));
            d = d + m->Xi[j] * (t * t) / sqrt(8.0 * (1.0 + m->Mi[i] / m->Mi[j]));
        }
        s = s + m->Xi[i] * r[i] / d;
    }
    return s;
}
double orc_mix_mu(const orc_mixture *m, double T) { return wilke(m, T, 1); }
double orc_mix_kp(const orc_mixture *m, double T) { return wilke(m, T, 0); }
double orc_mix_gm(const orc_mixture *m, double T)
{   /* :261-272 */
    double c = orc_mix_cp(m, T);
    return c / (c - m->Rg);
}

void orc_get_boundary_fields(int nx, int ny, const double *F, double *Fbn, double *Fbs, double *Fbe,
                             double *Fbw)
{   /* mod_field_operations.f90: east :3-26, west :29-52, north :62-84, south :88-110 */
    for (int i = 2; i <= nx - 1; i++) {
        Fbn[i - 1] = 0.5 * (F[IDX(i, ny - 1)] + F[IDX(i, ny)]);
        Fbs[i - 1] = 0.5 * (F[IDX(i, 2)] + F[IDX(i, 1)]);
    }
    for (int j = 2; j <= ny - 1; j++) {
        Fbe[j - 1] = 0.5 * (F[IDX(nx - 1, j)] + F[IDX(nx, j)]);
        Fbw[j - 1] = 0.5 * (F[IDX(2, j)] + F[IDX(1, j)]);
    }
}

void orc_set_cp(const orc_mixture *m, int nx, int ny, const double *Tbn, const double *Tbs, const double *Tbe,
                const double *Tbw, const double *T, double *cp)
{   /* mod_thermophysical.f90:79-218 */
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) cp[IDX(i, j)] = orc_mix_cp(m, T[IDX(i, j)]);
    for (int i = 2; i <= nx - 1; i++) cp[IDX(i, ny)] = orc_mix_cp(m, Tbn[i - 1]);
    for (int i = 2; i <= nx - 1; i++) cp[IDX(i, 1)] = orc_mix_cp(m, Tbs[i - 1]);
    for (int j = 2; j <= ny - 1; j++) cp[IDX(nx, j)] = orc_mix_cp(m, Tbe[j - 1]);
    for (int j = 2; j <= ny - 1; j++) cp[IDX(1, j)] = orc_mix_cp(m, Tbw[j - 1]);
    long np = IDX(1, 1);
    cp[np] = (cp[np + nx] + cp[np + 1] + cp[np + nx + 1]) / 3.0;
    np = IDX(nx, 1);
    cp[np] = (cp[np + nx] + cp[np - 1] + cp[np + nx - 1]) / 3.0;
    np = IDX(1, ny);
    cp[np] = (cp[np - nx] + cp[np + 1] + cp[np - nx + 1]) / 3.0;
    np = IDX(nx, ny);
    cp[np] = (cp[np - nx] + cp[np - 1] + cp[np - nx - 1]) / 3.0;
}

void orc_set_gamma(int nx, int ny, double Rg, const double *cp, double *gcp)
{   /* :223-235 */
    for (long k = 0; k < (long)nx * ny; k++) gcp[k] = cp[k] / (cp[k] - Rg);
}

void orc_transport_nodes(const orc_mixture *m, int nx, int ny, int visc, const double *T, double *phip)
{   /* set_laminar_viscosity_at_nodes :239-265, set_thermal_conductivity_at_nodes :269-295 */
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) phip[IDX(i, j)] = visc ? orc_mix_mu(m, T[IDX(i, j)]) : orc_mix_kp(m, T[IDX(i, j)]);
}

void orc_transport_faces(const orc_mixture *m, int nx, int ny, int visc, const double *Tbn, const double *Tbs,
                         const double *Tbe, const double *Tbw, const double *p, double *pe, double *pn)
{   /* get_laminar_viscosity_at_faces :299-402, get_thermal_conductivity_at_faces :406-509 */
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 2; i++) {
            long np = IDX(i, j);
            pe[np] = 2.0 * p[np] * p[np + 1] / (p[np] + p[np + 1]);
        }
    for (int j = 2; j <= ny - 1; j++) pe[IDX(1, j)] = visc ? orc_mix_mu(m, Tbw[j - 1]) : orc_mix_kp(m, Tbw[j - 1]);
    for (int j = 2; j <= ny - 1; j++)
        pe[IDX(nx - 1, j)] = visc ? orc_mix_mu(m, Tbe[j - 1]) : orc_mix_kp(m, Tbe[j - 1]);
    for (int i = 2; i <= nx - 1; i++)
        for (int j = 2; j <= ny - 2; j++) {
            long np = IDX(i, j);
            pn[np] = 2.0 * p[np] * p[np + nx] / (p[np] + p[np + nx]);
        }
    for (int i = 2; i <= nx - 1; i++) pn[IDX(i, 1)] = visc ? orc_mix_mu(m, Tbs[i - 1]) : orc_mix_kp(m, Tbs[i - 1]);
    for (int i = 2; i <= nx - 1; i++)
        pn[IDX(i, ny - 1)] = visc ? orc_mix_mu(m, Tbn[i - 1]) : orc_mix_kp(m, Tbn[i - 1]);
}
