// m2d_stencil.cu -- FP64 stencil kernels of one SIMPLEC outer iteration.
//
// One thread per cell (or per face / boundary cell), 32x8 blocks, so each warp
// reads 32 consecutive cells of a row from every plane: HBM-bound kernels
// with fully coalesced 256-byte transactions.  Every kernel restates one
// reference routine (cited per kernel) with the same per-cell expression in
// the same evaluation order; with -fmad=false the results are bitwise equal
// to a sequential FP64 evaluation.
#include "m2d_fields.cuh"

namespace m2d {

#define IDX(i, j) ((long long)((j) - 1) * nx + ((i) - 1))
#define A9(a, np, k) (a)[(long long)((k) - 1) * N + (np)]

static inline dim3 grid2d(int nx, int ny)
{
    return dim3((unsigned)((nx + 31) / 32), (unsigned)((ny + 7) / 8));
}
#define CELL_IJ                                    \
    const int i = blockIdx.x * 32 + threadIdx.x + 1; \
    const int j = blockIdx.y * 8 + threadIdx.y + 1;
static const dim3 kBlock2d(32, 8);

// ---------------------------------------------------------------------------
// get_density_at_nodes  src/equations/mach2d_coef.f90:6-17
__global__ void k_density_nodes(Fields f, double Rg)
{
    long long N = (long long)f.nx * f.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N;
         k += (long long)gridDim.x * blockDim.x)
        f.ro[k] = f.p[k] / (Rg * f.T[k]);
}

// get_density_at_faces  src/equations/mach2d_coef.f90:20-60
__global__ void k_density_faces(Fields f, double beta)
{
    const int nx = f.nx, ny = f.ny;
    CELL_IJ
    if (i > nx || j > ny) return;
    long long np = IDX(i, j);
    if (j >= 2 && j <= ny - 1 && i <= nx - 1) {
        long long npe = np + 1;
        double ae = sgn05(f.Uce[np]);
        f.roe[np] = (0.5 + ae) * f.ro[np] + (0.5 - ae) * f.ro[npe] + beta * ae * (f.ro[npe] - f.ro[np]);
    }
    if (j <= ny - 1 && i >= 2 && i <= nx - 1) {
        long long npn = np + nx;
        double an = sgn05(f.Vcn[np]);
        f.ron[np] = (0.5 + an) * f.ro[np] + (0.5 - an) * f.ro[npn] + beta * an * (f.ro[npn] - f.ro[np]);
    }
}

// ---------------------------------------------------------------------------
// get_u_coefficients + get_u_source  src/equations/mach2d_coef.f90:63-451
__device__ __forceinline__ void u_assembly_cell(const Fields &f, const Params &q, int what, int i, int j)
{
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j), nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    const double *roe = f.roe, *ron = f.ron, *re = f.re, *rn = f.rn, *Uce = f.Uce, *Vcn = f.Vcn;
    const double fme = roe[np] * re[np] * Uce[np];
    const double fmw = roe[npw] * re[npw] * Uce[npw];
    const double fmn = ron[np] * rn[np] * Vcn[np];
    const double fms = ron[nps] * rn[nps] * Vcn[nps];
    const double mpa = f.roa[np] * f.rp[np] / f.Jp[np];
    const double as = sgn05(Vcn[nps]), an = sgn05(Vcn[np]);
    const double aw = sgn05(Uce[npw]), ae = sgn05(Uce[np]);
    const double dt = q.dtp ? *q.dtp : q.dt;
    if (what & ASM_COEF) {
        double *a = f.au;
        if (q.modvis == 0) {
            double a2 = -fms * (0.5 + as), a4 = -fmw * (0.5 + aw);
            double a6 = fme * (0.5 - ae), a8 = fmn * (0.5 - an);
            A9(a, np, 1) = 0.0; A9(a, np, 3) = 0.0; A9(a, np, 7) = 0.0; A9(a, np, 9) = 0.0;
            A9(a, np, 2) = a2; A9(a, np, 4) = a4; A9(a, np, 6) = a6; A9(a, np, 8) = a8;
            A9(a, np, 5) = mpa / dt - (a8 + a2 + a4 + a6);
        } else {
            const double *vle = f.vle, *vln = f.vln, *Je = f.Je, *Jn = f.Jn;
            const double *betae = f.betae, *betan = f.betan, *alphae = f.alphae, *gamman = f.gamman;
            const double *ye = f.ye, *yk = f.yk, *rp = f.rp;
            double a1 = (vle[npw] * re[npw] * Je[npw] * betae[npw] + vln[nps] * rn[nps] * Jn[nps] * betan[nps]) / 4.0;
            double a2 = -fms * (0.5 + as) - vln[nps] * rn[nps] * Jn[nps] * gamman[nps]
                      + (vle[npw] * re[npw] * Je[npw] * betae[npw] - vle[np] * re[np] * Je[np] * betae[np]) / 4.0;
            double a3 = -(vle[np] * re[np] * Je[np] * betae[np] + vln[nps] * rn[nps] * Jn[nps] * betan[nps]) / 4.0;
            double a4 = -fmw * (0.5 + aw) - vle[npw] * re[npw] * Je[npw] * alphae[npw]
                      + (vln[nps] * rn[nps] * Jn[nps] * betan[nps] - vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a6 = fme * (0.5 - ae) - vle[np] * re[np] * Je[np] * alphae[np]
                      + (-vln[nps] * rn[nps] * Jn[nps] * betan[nps] + vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a7 = (-vle[npw] * re[npw] * Je[npw] * betae[npw] - vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a8 = fmn * (0.5 - an) - vln[np] * rn[np] * Jn[np] * gamman[np]
                      - (vle[npw] * re[npw] * Je[npw] * betae[npw] - vle[np] * re[np] * Je[np] * betae[np]) / 4.0;
            double a9 = (vle[np] * re[np] * Je[np] * betae[np] + vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a5 = mpa / dt - (a8 + a2 + a4 + a6);
            double S1p = rp[np] * Je[np] * vle[np] * (ye[np] * ye[np]) / 3.0
                       + rp[np] * Je[npw] * vle[npw] * (ye[npw] * ye[npw]) / 3.0;
            double S2p = rp[np] * Jn[np] * vln[np] * (yk[np] * yk[np]) / 3.0
                       + rp[np] * Jn[nps] * vln[nps] * (yk[nps] * yk[nps]) / 3.0;
            a5 = a5 + S1p + S2p;
            A9(a, np, 1) = a1; A9(a, np, 2) = a2; A9(a, np, 3) = a3; A9(a, np, 4) = a4; A9(a, np, 5) = a5;
            A9(a, np, 6) = a6; A9(a, np, 7) = a7; A9(a, np, 8) = a8; A9(a, np, 9) = a9;
        }
    }
    if (!(what & ASM_SRC)) return;
    const double *u = f.u, *v = f.v, *p = f.p, *rp = f.rp, *ye = f.ye, *yk = f.yk;
    double b = mpa * f.ua[np] / dt;
    double cup = -(q.beta * (fme * ae * (u[npe] - u[np]) - fmw * aw * (u[np] - u[npw])
                             + fmn * an * (u[npn] - u[np]) - fms * as * (u[np] - u[nps])));
    b = b + cup;
    b = b + 0.5 * rp[np] * (+yk[np] * (p[npn] + p[np]) - yk[nps] * (p[nps] + p[np])
                            - ye[np] * (p[npe] + p[np]) + ye[npw] * (p[npw] + p[np]));
    f.cup[np] = cup;
    if (q.modvis == 1) {
        const long long npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
        const double *Je = f.Je, *Jn = f.Jn, *vle = f.vle, *vln = f.vln, *xe = f.xe, *xk = f.xk;
        const double *xke = f.xke, *yke = f.yke, *xen = f.xen, *yen = f.yen;
        double S1, S2, S3, S4, S5, S6;
        S1 = rp[np] / 3.0 * (+Je[np] * vle[np] * ((ye[np] * ye[np]) * u[npe] - yke[np] * ye[np] * (u[npn] + u[npne] - u[nps] - u[npse]) / 4.0)
                             - Je[npw] * vle[npw] * (-(ye[npw] * ye[npw]) * u[npw] - yke[npw] * ye[npw] * (u[npn] + u[npnw] - u[nps] - u[npsw]) / 4.0));
        S2 = rp[np] / 3.0 * (+Jn[np] * vln[np] * ((yk[np] * yk[np]) * u[npn] - yk[np] * yen[np] * (u[npe] + u[npne] - u[npw] - u[npnw]) / 4.0)
                             - Jn[nps] * vln[nps] * (-(yk[nps] * yk[nps]) * u[nps] - yk[nps] * yen[nps] * (u[npe] + u[npse] - u[npw] - u[npsw]) / 4.0));
        S3 = Je[np] * re[np] * vle[np] * xe[np] * (yke[np] * (v[npn] + v[npne] - v[nps] - v[npse]) / 4.0 - ye[np] * (v[npe] - v[np]))
           - Je[npw] * re[npw] * vle[npw] * xe[npw] * (yke[npw] * (v[npn] + v[npnw] - v[nps] - v[npsw]) / 4.0 - ye[npw] * (v[np] - v[npw]));
        S4 = Jn[np] * rn[np] * vln[np] * xk[np] * (yen[np] * (v[npne] + v[npe] - v[npnw] - v[npw]) / 4.0 - yk[np] * (v[npn] - v[np]))
           - Jn[nps] * rn[nps] * vln[nps] * xk[nps] * (yen[nps] * (v[npse] + v[npe] - v[npsw] - v[npw]) / 4.0 - yk[nps] * (v[np] - v[nps]));
        double t5e = 2.0 * rp[np] / 3.0 * Je[np] * vle[np] / re[np] * ye[np]
                   * (xke[np] * (rp[npn] * v[npn] + rp[npne] * v[npne] - rp[nps] * v[nps] - rp[npse] * v[npse]) / 4.0
                      - xe[np] * (rp[npe] * v[npe] - rp[np] * v[np]));
        double t5w = 2.0 * rp[np] / 3.0 * Je[npw] * vle[npw] / re[npw] * ye[npw]
                   * (xke[npw] * (rp[npn] * v[npn] + rp[npnw] * v[npnw] - rp[nps] * v[nps] - rp[npsw] * v[npsw]) / 4.0
                      - xe[npw] * (rp[np] * v[np] - rp[npw] * v[npw]));
        if (fabs(re[npw]) < 1.0e-15) S5 = -t5e;
        else if (fabs(re[np]) < 1.0e-15) S5 = +t5w;
        else S5 = -t5e + t5w;
        double t6n = 2.0 * rp[np] / 3.0 * Jn[np] * vln[np] / rn[np] * yk[np]
                   * (xen[np] * (rp[npne] * v[npne] + rp[npe] * v[npe] - rp[npnw] * v[npnw] - rp[npw] * v[npw]) / 4.0
                      - xk[np] * (rp[npn] * v[npn] - rp[np] * v[np]));
        double t6s = 2.0 * rp[np] / 3.0 * Jn[nps] * vln[nps] / rn[nps] * yk[nps]
                   * (xen[nps] * (rp[npe] * v[npe] + rp[npse] * v[npse] - rp[npw] * v[npw] - rp[npsw] * v[npsw]) / 4.0
                      - xk[nps] * (rp[np] * v[np] - rp[nps] * v[nps]));
        if (fabs(rn[nps]) < 1.0e-15) S6 = -t6n;
        else if (fabs(rn[np]) < 1.0e-15) S6 = t6s;
        else S6 = -t6n + t6s;
        double sup = S1 + S2 + S3 + S4 + S5 + S6;
        f.sup[np] = sup;
        b = b + sup;
    }
    f.bu[np] = b;
}
__global__ void k_u_assembly(Fields f, Params q, int what)
{
    CELL_IJ
    u_assembly_cell(f, q, what, i, j);
}

// get_v_coefficients + get_v_source  src/equations/mach2d_coef.f90:454-783
__device__ __forceinline__ void v_assembly_cell(const Fields &f, const Params &q, int what, int i, int j)
{
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j), nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    const double *roe = f.roe, *ron = f.ron, *re = f.re, *rn = f.rn, *Uce = f.Uce, *Vcn = f.Vcn;
    const double fme = roe[np] * re[np] * Uce[np];
    const double fmw = roe[npw] * re[npw] * Uce[npw];
    const double fmn = ron[np] * rn[np] * Vcn[np];
    const double fms = ron[nps] * rn[nps] * Vcn[nps];
    const double mpa = f.roa[np] * f.rp[np] / f.Jp[np];
    const double as = sgn05(Vcn[nps]), an = sgn05(Vcn[np]);
    const double aw = sgn05(Uce[npw]), ae = sgn05(Uce[np]);
    const double dt = q.dtp ? *q.dtp : q.dt;
    if (what & ASM_COEF) {
        double *a = f.av;
        if (q.modvis == 0) {
            double a2 = -fms * (0.5 + as), a4 = -fmw * (0.5 + aw);
            double a6 = fme * (0.5 - ae), a8 = fmn * (0.5 - an);
            A9(a, np, 1) = 0.0; A9(a, np, 3) = 0.0; A9(a, np, 7) = 0.0; A9(a, np, 9) = 0.0;
            A9(a, np, 2) = a2; A9(a, np, 4) = a4; A9(a, np, 6) = a6; A9(a, np, 8) = a8;
            A9(a, np, 5) = mpa / dt - (a8 + a2 + a4 + a6);
        } else {
            const double *vle = f.vle, *vln = f.vln, *Je = f.Je, *Jn = f.Jn;
            const double *betae = f.betae, *betan = f.betan, *alphae = f.alphae, *gamman = f.gamman;
            const double *xe = f.xe, *xk = f.xk, *rp = f.rp;
            double a1 = (vle[npw] * re[npw] * Je[npw] * betae[npw] + vln[nps] * rn[nps] * Jn[nps] * betan[nps]) / 4.0;
            double a2 = -fms * (0.5 + as) - vln[nps] * rn[nps] * Jn[nps] * gamman[nps]
                      + (vle[npw] * re[npw] * Je[npw] * betae[npw] - vle[np] * re[np] * Je[np] * betae[np]) / 4.0;
            double a3 = -(vle[np] * re[np] * Je[np] * betae[np] + vln[nps] * rn[nps] * Jn[nps] * betan[nps]) / 4.0;
            double a4 = -fmw * (0.5 + aw) - vle[npw] * re[npw] * Je[npw] * alphae[npw]
                      + (vln[nps] * rn[nps] * Jn[nps] * betan[nps] - vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a6 = fme * (0.5 - ae) - vle[np] * re[np] * Je[np] * alphae[np]
                      + (-vln[nps] * rn[nps] * Jn[nps] * betan[nps] + vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a7 = (-vle[npw] * re[npw] * Je[npw] * betae[npw] - vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a8 = fmn * (0.5 - an) - vln[np] * rn[np] * Jn[np] * gamman[np]
                      - (vle[npw] * re[npw] * Je[npw] * betae[npw] - vle[np] * re[np] * Je[np] * betae[np]) / 4.0;
            double a9 = (vle[np] * re[np] * Je[np] * betae[np] + vln[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
            double a5 = mpa / dt - (a8 + a2 + a4 + a6);
            double S1p = vle[np] * re[np] * Je[np] * (xe[np] * xe[np]) / 3.0
                       + vle[npw] * re[npw] * Je[npw] * (xe[npw] * xe[npw]) / 3.0;
            double S2p = vln[np] * rn[np] * Jn[np] * (xk[np] * xk[np]) / 3.0
                       + vln[nps] * rn[nps] * Jn[nps] * (xk[nps] * xk[nps]) / 3.0;
            double S7p = (double)q.coord * f.vlp[np] * 4.0 / (3.0 * rp[np] * f.Jp[np]);
            a5 = a5 + S1p + S2p + S7p;
            A9(a, np, 1) = a1; A9(a, np, 2) = a2; A9(a, np, 3) = a3; A9(a, np, 4) = a4; A9(a, np, 5) = a5;
            A9(a, np, 6) = a6; A9(a, np, 7) = a7; A9(a, np, 8) = a8; A9(a, np, 9) = a9;
        }
    }
    if (!(what & ASM_SRC)) return;
    const double *u = f.u, *v = f.v, *p = f.p, *rp = f.rp, *xe = f.xe, *xk = f.xk;
    double b = mpa * f.va[np] / dt;
    double cvp = -(q.beta * (fme * ae * (v[npe] - v[np]) - fmw * aw * (v[np] - v[npw])
                             + fmn * an * (v[npn] - v[np]) - fms * as * (v[np] - v[nps])));
    b = b + cvp;
    b = b + 0.5 * rp[np] * (+xe[np] * (p[np] + p[npe]) - xe[npw] * (p[np] + p[npw])
                            - xk[np] * (p[np] + p[npn]) + xk[nps] * (p[np] + p[nps]));
    f.cvp[np] = cvp;
    if (q.modvis == 1) {
        const long long npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
        const double *Je = f.Je, *Jn = f.Jn, *vle = f.vle, *vln = f.vln, *ye = f.ye, *yk = f.yk;
        const double *xke = f.xke, *yke = f.yke, *xen = f.xen, *yen = f.yen;
        double S1, S2, S3, S4, S5, S6, S8;
        S1 = vle[np] * re[np] * Je[np] / 3.0 * ((xe[np] * xe[np]) * v[npe] - xke[np] * xe[np] * (v[npn] + v[npne] - v[nps] - v[npse]) / 4.0)
           - vle[npw] * re[npw] * Je[npw] / 3.0 * (-(xe[npw] * xe[npw]) * v[npw] - xke[npw] * xe[npw] * (v[npn] + v[npnw] - v[nps] - v[npsw]) / 4.0);
        S2 = vln[np] * rn[np] * Jn[np] / 3.0 * ((xk[np] * xk[np]) * v[npn] - xk[np] * xen[np] * (v[npe] + v[npne] - v[npnw] - v[npw]) / 4.0)
           - vln[nps] * rn[nps] * Jn[nps] / 3.0 * (-(xk[nps] * xk[nps]) * v[nps] - xk[nps] * xen[nps] * (v[npe] + v[npse] - v[npsw] - v[npw]) / 4.0);
        S3 = rp[np] * vle[np] * Je[np] * ye[np] * (+xke[np] * (u[npn] + u[npne] - u[nps] - u[npse]) / 4.0 - xe[np] * (u[npe] - u[np]))
           - rp[np] * vle[npw] * Je[npw] * ye[npw] * (+xke[npw] * (u[npn] + u[npnw] - u[nps] - u[npsw]) / 4.0 - xe[npw] * (u[np] - u[npw]));
        S4 = rp[np] * vln[np] * Jn[np] * yk[np] * (+xen[np] * (u[npne] + u[npe] - u[npnw] - u[npw]) / 4.0 - xk[np] * (u[npn] - u[np]))
           - rp[np] * vln[nps] * Jn[nps] * yk[nps] * (+xen[nps] * (u[npse] + u[npe] - u[npsw] - u[npw]) / 4.0 - xk[nps] * (u[np] - u[nps]));
        S5 = -(2.0 / 3.0 * rp[np] * vle[np] * Je[np] * xe[np] * (+yke[np] * (u[npn] + u[npne] - u[nps] - u[npse]) / 4.0 - ye[np] * (u[npe] - u[np])))
           + 2.0 / 3.0 * rp[np] * vle[npw] * Je[npw] * xe[npw] * (+yke[npw] * (u[npn] + u[npnw] - u[nps] - u[npsw]) / 4.0 - ye[npw] * (u[np] - u[npw]));
        S6 = -(2.0 / 3.0 * rp[np] * vln[np] * Jn[np] * xk[np] * (+yen[np] * (u[npe] + u[npne] - u[npw] - u[npnw]) / 4.0 - yk[np] * (u[npn] - u[np])))
           + 2.0 / 3.0 * rp[np] * vln[nps] * Jn[nps] * xk[nps] * (+yen[nps] * (u[npe] + u[npse] - u[npw] - u[npsw]) / 4.0 - yk[nps] * (u[np] - u[nps]));
        S8 = 2.0 / 3.0 * (double)q.coord * v[np] * (-vln[np] * xk[np] + vln[nps] * xk[nps] + vle[np] * xe[np] - vle[npw] * xe[npw]);
        double svp = S1 + S2 + S3 + S4 + S5 + S6 + S8;
        f.svp[np] = svp;
        b = b + svp;
    }
    f.bv[np] = b;
}
__global__ void k_v_assembly(Fields f, Params q, int what)
{
    CELL_IJ
    v_assembly_cell(f, q, what, i, j);
}

// get_T_coefficients_and_source  src/equations/mach2d_coef.f90:787-1203
__global__ void k_T_assembly(Fields f, Params q)
{
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    CELL_IJ
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j), nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    const long long npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
    const double *roe = f.roe, *ron = f.ron, *re = f.re, *rn = f.rn, *Uce = f.Uce, *Vcn = f.Vcn;
    const double *cp = f.cp, *u = f.u, *v = f.v, *T = f.T, *rp = f.rp, *Jp = f.Jp;
    const double beta = q.beta, dt = q.dtp ? *q.dtp : q.dt, eps = 2.220446049250313e-16;
    const double fme = roe[np] * re[np] * Uce[np];
    const double fmw = roe[npw] * re[npw] * Uce[npw];
    const double fmn = ron[np] * rn[np] * Vcn[np];
    const double fms = ron[nps] * rn[nps] * Vcn[nps];
    const double mpa = f.roa[np] * rp[np] / Jp[np];
    const double as = sgn05(Vcn[nps]), an = sgn05(Vcn[np]);
    const double aw = sgn05(Uce[npw]), ae = sgn05(Uce[np]);
    double a1, a2, a3, a4, a6, a7, a8, a9;
    if (q.modvis == 0) {
        a1 = 0.0; a3 = 0.0; a7 = 0.0; a9 = 0.0;
        a2 = -fms * (0.5 + as) * cp[np];
        a4 = -fmw * (0.5 + aw) * cp[np];
        a6 = fme * (0.5 - ae) * cp[np];
        a8 = fmn * (0.5 - an) * cp[np];
    } else {
        const double *ke = f.ke, *kn = f.kn, *Je = f.Je, *Jn = f.Jn;
        const double *betae = f.betae, *betan = f.betan, *alphae = f.alphae, *gamman = f.gamman;
        a1 = (ke[npw] * re[npw] * Je[npw] * betae[npw] + kn[nps] * rn[nps] * Jn[nps] * betan[nps]) / 4.0;
        a2 = -fms * (0.5 + as) * cp[np] - kn[nps] * rn[nps] * Jn[nps] * gamman[nps]
           + (ke[npw] * re[npw] * Je[npw] * betae[npw] - ke[np] * re[np] * Je[np] * betae[np]) / 4.0;
        a3 = -(ke[np] * re[np] * Je[np] * betae[np] + kn[nps] * rn[nps] * Jn[nps] * betan[nps]) / 4.0;
        a4 = -fmw * (0.5 + aw) * cp[np] - ke[npw] * re[npw] * Je[npw] * alphae[npw]
           + (kn[nps] * rn[nps] * Jn[nps] * betan[nps] - kn[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
        a6 = fme * (0.5 - ae) * cp[np] - ke[np] * re[np] * Je[np] * alphae[np]
           + (-kn[nps] * rn[nps] * Jn[nps] * betan[nps] + kn[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
        a7 = (-ke[npw] * re[npw] * Je[npw] * betae[npw] - kn[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
        a8 = fmn * (0.5 - an) * cp[np] - kn[np] * rn[np] * Jn[np] * gamman[np]
           - (ke[npw] * re[npw] * Je[npw] * betae[npw] - ke[np] * re[np] * Je[np] * betae[np]) / 4.0;
        a9 = (ke[np] * re[np] * Je[np] * betae[np] + kn[np] * rn[np] * Jn[np] * betan[np]) / 4.0;
    }
    double *a = f.at;
    A9(a, np, 1) = a1; A9(a, np, 2) = a2; A9(a, np, 3) = a3; A9(a, np, 4) = a4;
    A9(a, np, 5) = mpa * cp[np] / dt - (a8 + a2 + a4 + a6);
    A9(a, np, 6) = a6; A9(a, np, 7) = a7; A9(a, np, 8) = a8; A9(a, np, 9) = a9;
    double b = mpa * f.Ta[np] * cp[np] / dt;
    b = b - beta * cp[np] * (fme * ae * (T[npe] - T[np]) - fmw * aw * (T[np] - T[npw])
                             + fmn * an * (T[npn] - T[np]) - fms * as * (T[np] - T[nps]));
    const double *ue = f.ue, *ve = f.ve, *un = f.un, *vn = f.vn, *ua = f.ua, *va = f.va;
    double KpE = (u[npe] * u[npe] + v[npe] * v[npe]) / 2.0;
    double KpW = (u[npw] * u[npw] + v[npw] * v[npw]) / 2.0;
    double KpN = (u[npn] * u[npn] + v[npn] * v[npn]) / 2.0;
    double KpS = (u[nps] * u[nps] + v[nps] * v[nps]) / 2.0;
    double KpP = (u[np] * u[np] + v[np] * v[np]) / 2.0;
    double KpPa = (ua[np] * ua[np] + va[np] * va[np]) / 2.0;
    double Kfe = (0.5 + ae) * KpP + (0.5 - ae) * KpE + beta * ae * (KpE - KpP);
    double Kfw = (0.5 + aw) * KpW + (0.5 - aw) * KpP + beta * aw * (KpP - KpW);
    double Kfn = (0.5 + an) * KpP + (0.5 - an) * KpN + beta * an * (KpN - KpP);
    double Kfs = (0.5 + as) * KpS + (0.5 - as) * KpP + beta * as * (KpP - KpS);
    double Kfbe = (ue[np] * ue[np] + ve[np] * ve[np]) / 2.0;
    double Kfbw = (ue[npw] * ue[npw] + ve[npw] * ve[npw]) / 2.0;
    double Kfbn = (un[np] * un[np] + vn[np] * vn[np]) / 2.0;
    double Kfbs = (un[nps] * un[nps] + vn[nps] * vn[nps]) / 2.0;
    const double *fbe = f.fbe, *fbn = f.fbn;
    Kfe = Kfe * (1.0 - fbe[np]) + Kfbe * fbe[np];
    Kfw = Kfw * (1.0 - fbe[npw]) + Kfbw * fbe[npw];
    Kfn = Kfn * (1.0 - fbn[np]) + Kfbn * fbn[np];
    Kfs = Kfs * (1.0 - fbn[nps]) + Kfbs * fbn[nps];
    double raux = rp[np] / Jp[np] * (f.ro[np] * KpP - f.roa[np] * KpPa) / dt
                + fme * Kfe - fmw * Kfw + fmn * Kfn - fms * Kfs;
    b = b + rp[np] / Jp[np] * (f.p[np] - f.pa[np]) / dt - raux;
    if (q.modvis != 0) {
        const double *Je = f.Je, *Jn = f.Jn, *xe = f.xe, *ye = f.ye, *xk = f.xk, *yk = f.yk;
        const double *xke = f.xke, *yke = f.yke, *xen = f.xen, *yen = f.yen, *vle = f.vle, *vln = f.vln;
        double dudk_e = u[npe] - u[np], dudk_w = u[np] - u[npw];
        double dudk_n = (u[npne] + u[npe] - u[npnw] - u[npw]) / 4.0;
        double dudk_s = (u[npse] + u[npe] - u[npsw] - u[npw]) / 4.0;
        double dude_e = (u[npne] + u[npn] - u[npse] - u[nps]) / 4.0;
        double dude_w = (u[npnw] + u[npn] - u[npsw] - u[nps]) / 4.0;
        double dude_n = u[npn] - u[np], dude_s = u[np] - u[nps];
        double dvdk_e = v[npe] - v[np], dvdk_w = v[np] - v[npw];
        double dvdk_n = (v[npne] + v[npe] - v[npnw] - v[npw]) / 4.0;
        double dvdk_s = (v[npse] + v[npe] - v[npsw] - v[npw]) / 4.0;
        double dvde_e = (v[npne] + v[npn] - v[npse] - v[nps]) / 4.0;
        double dvde_w = (v[npnw] + v[npn] - v[npsw] - v[nps]) / 4.0;
        double dvde_n = v[npn] - v[np], dvde_s = v[np] - v[nps];
        double dudx_e = Je[np] * (ye[np] * dudk_e - yke[np] * dude_e);
        double dudx_w = Je[npw] * (ye[npw] * dudk_w - yke[npw] * dude_w);
        double dudx_n = Jn[np] * (yen[np] * dudk_n - yk[np] * dude_n);
        double dudx_s = Jn[nps] * (yen[nps] * dudk_s - yk[nps] * dude_s);
        double dudy_e = Je[np] * (xke[np] * dude_e - xe[np] * dudk_e);
        double dudy_w = Je[npw] * (xke[npw] * dude_w - xe[npw] * dudk_w);
        double dudy_n = Jn[np] * (xk[np] * dude_n - xen[np] * dudk_n);
        double dudy_s = Jn[nps] * (xk[nps] * dude_s - xen[nps] * dudk_s);
        double dvdx_e = Je[np] * (ye[np] * dvdk_e - yke[np] * dvde_e);
        double dvdx_w = Je[npw] * (ye[npw] * dvdk_w - yke[npw] * dvde_w);
        double dvdx_n = Jn[np] * (yen[np] * dvdk_n - yk[np] * dvde_n);
        double dvdx_s = Jn[nps] * (yen[nps] * dvdk_s - yk[nps] * dvde_s);
        double dvdy_e = Je[np] * (xke[np] * dvde_e - xe[np] * dvdk_e);
        double dvdy_w = Je[npw] * (xke[npw] * dvde_w - xe[npw] * dvdk_w);
        double dvdy_n = Jn[np] * (xk[np] * dvde_n - xen[np] * dvdk_n);
        double dvdy_s = Jn[nps] * (xk[nps] * dvde_s - xen[nps] * dvdk_s);
        double divU_e = dudx_e + dvdy_e + ve[np] / (fabs(re[np]) + eps);
        double divU_w = dudx_w + dvdy_w + ve[npw] / (fabs(re[npw]) + eps);
        double divU_n = dudx_n + dvdy_n + vn[np] / (fabs(rn[np]) + eps);
        double divU_s = dudx_s + dvdy_s + vn[nps] / (fabs(rn[nps]) + eps);
        double Txx_e = -2.0 * vle[np] * dudx_e + 2.0 / 3.0 * vle[np] * divU_e;
        double Txx_w = -2.0 * vle[npw] * dudx_w + 2.0 / 3.0 * vle[npw] * divU_w;
        double Txx_n = -2.0 * vln[np] * dudx_n + 2.0 / 3.0 * vln[np] * divU_n;
        double Txx_s = -2.0 * vln[nps] * dudx_s + 2.0 / 3.0 * vln[nps] * divU_s;
        double Txy_e = -(vle[np] * (dvdx_e + dudy_e));
        double Txy_w = -(vle[npw] * (dvdx_w + dudy_w));
        double Txy_n = -(vln[np] * (dvdx_n + dudy_n));
        double Txy_s = -(vln[nps] * (dvdx_s + dudy_s));
        double Tyy_e = -2.0 * vle[np] * dvdy_e + 2.0 / 3.0 * vle[np] * divU_e;
        double Tyy_w = -2.0 * vle[npw] * dvdy_w + 2.0 / 3.0 * vle[npw] * divU_w;
        double Tyy_n = -2.0 * vln[np] * dvdy_n + 2.0 / 3.0 * vln[np] * divU_n;
        double Tyy_s = -2.0 * vln[nps] * dvdy_s + 2.0 / 3.0 * vln[nps] * divU_s;
        double Lbd_x_e = ve[np] * Txy_e + ue[np] * Txx_e;
        double Lbd_x_w = ve[npw] * Txy_w + ue[npw] * Txx_w;
        double Lbd_x_n = vn[np] * Txy_n + un[np] * Txx_n;
        double Lbd_x_s = vn[nps] * Txy_s + un[nps] * Txx_s;
        double Lbd_y_e = ve[np] * Tyy_e + ue[np] * Txy_e;
        double Lbd_y_w = ve[npw] * Tyy_w + ue[npw] * Txy_w;
        double Lbd_y_n = vn[np] * Tyy_n + un[np] * Txy_n;
        double Lbd_y_s = vn[nps] * Tyy_s + un[nps] * Txy_s;
        double Lbd_k_e = Lbd_x_e * ye[np] - Lbd_y_e * xe[np];
        double Lbd_k_w = Lbd_x_w * ye[npw] - Lbd_y_w * xe[npw];
        double Lbd_e_n = Lbd_y_n * xk[np] - Lbd_x_n * yk[np];
        double Lbd_e_s = Lbd_y_s * xk[nps] - Lbd_x_s * yk[nps];
        raux = re[np] * Lbd_k_e - re[npw] * Lbd_k_w + rn[np] * Lbd_e_n - rn[nps] * Lbd_e_s;
        b = b - raux;
    }
    f.bt[np] = b;
}

// get_p_coefficients + get_p_source  src/equations/mach2d_coef.f90:1207-1348
__device__ __forceinline__ void p_assembly_cell(const Fields &f, const Params &q, int what, int i, int j)
{
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    if (q.maxpl && (what & ASM_COEF) && i == 1 && j == 1) *q.maxpl = 0.0;   // k_p_cycle_update's max|p'|
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j), nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    const double *re = f.re, *rn = f.rn, *Uce = f.Uce, *Vcn = f.Vcn, *g = f.g;
    const double *de = f.de, *dn = f.dn, *roe = f.roe, *ron = f.ron;
    const double dt = q.dtp ? *q.dtp : q.dt;
    const double as = sgn05(Vcn[nps]), an = sgn05(Vcn[np]);
    const double aw = sgn05(Uce[npw]), ae = sgn05(Uce[np]);
    if (what & ASM_COEF) {
        const double roem = roe[np], rowm = roe[npw], ronm = ron[np], rosm = ron[nps];
        double *a = f.ap;
        A9(a, np, 1) = -(rn[nps] * ((0.5 + as) * Vcn[nps] * g[nps] + rosm * dn[nps]));
        A9(a, np, 2) = -(re[npw] * ((0.5 + aw) * Uce[npw] * g[npw] + rowm * de[npw]));
        A9(a, np, 3) = g[np] * (f.rp[np] / (f.Jp[np] * dt) + (0.5 + ae) * re[np] * Uce[np]
                                - (0.5 - aw) * re[npw] * Uce[npw] + (0.5 + an) * rn[np] * Vcn[np]
                                - (0.5 - as) * rn[nps] * Vcn[nps])
                     + roem * re[np] * de[np] + rowm * re[npw] * de[npw]
                     + ronm * rn[np] * dn[np] + rosm * rn[nps] * dn[nps];
        A9(a, np, 4) = re[np] * ((0.5 - ae) * Uce[np] * g[npe] - roem * de[np]);
        A9(a, np, 5) = rn[np] * ((0.5 - an) * Vcn[np] * g[npn] - ronm * dn[np]);
    }
    if (what & ASM_SRC) {
        const double *pl = f.pl;
        double roel = g[np] * pl[np] * (0.5 + ae) + g[npe] * pl[npe] * (0.5 - ae);
        double rowl = g[npw] * pl[npw] * (0.5 + aw) + g[np] * pl[np] * (0.5 - aw);
        double ronl = g[np] * pl[np] * (0.5 + an) + g[npn] * pl[npn] * (0.5 - an);
        double rosl = g[nps] * pl[nps] * (0.5 + as) + g[np] * pl[np] * (0.5 - as);
        double Ucel = de[np] * (pl[np] - pl[npe]);
        double Ucwl = de[npw] * (pl[npw] - pl[np]);
        double Vcnl = dn[np] * (pl[np] - pl[npn]);
        double Vcsl = dn[nps] * (pl[nps] - pl[np]);
        f.bp[np] = -f.rp[np] * (f.ro[np] - f.roa[np]) / (f.Jp[np] * dt)
                 - roe[np] * re[np] * Uce[np] + roe[npw] * re[npw] * Uce[npw]
                 - ron[np] * rn[np] * Vcn[np] + ron[nps] * rn[nps] * Vcn[nps]
                 - roel * re[np] * Ucel + rowl * re[npw] * Ucwl
                 - ronl * rn[np] * Vcnl + rosl * rn[nps] * Vcsl;
    }
}
__global__ void k_p_assembly(Fields f, Params q, int what)
{
    CELL_IJ
    p_assembly_cell(f, q, what, i, j);
}

// get_velocities_at_internal_faces  src/equations/mach2d_coef.f90:1350-1501
__device__ __forceinline__ void faces_internal_cell(const Fields &f, double dt, const double *dtp, int i, int j)
{
    if (dtp) dt = *dtp;
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j), nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    const long long npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
    const double *au = f.au, *av = f.av, *u = f.u, *v = f.v, *p = f.p;
    const double mpa = f.roa[np] * f.rp[np] / f.Jp[np];
    const double sumup = A9(au, np, 1) * u[npsw] + A9(au, np, 2) * u[nps] + A9(au, np, 3) * u[npse]
                       + A9(au, np, 4) * u[npw] + A9(au, np, 6) * u[npe] + A9(au, np, 7) * u[npnw]
                       + A9(au, np, 8) * u[npn] + A9(au, np, 9) * u[npne];
    const double sumvp = A9(av, np, 1) * v[npsw] + A9(av, np, 2) * v[nps] + A9(av, np, 3) * v[npse]
                       + A9(av, np, 4) * v[npw] + A9(av, np, 6) * v[npe] + A9(av, np, 7) * v[npnw]
                       + A9(av, np, 8) * v[npn] + A9(av, np, 9) * v[npne];
    if (i <= nx - 2) {
        const long long npee = npe + 1, npsee = npse + 1, npnee = npne + 1;
        const double mea = f.roa[npe] * f.rp[npe] / f.Jp[npe];
        double sumue = A9(au, npe, 1) * u[nps] + A9(au, npe, 2) * u[npse] + A9(au, npe, 3) * u[npsee]
                     + A9(au, npe, 4) * u[np] + A9(au, npe, 6) * u[npee] + A9(au, npe, 7) * u[npn]
                     + A9(au, npe, 8) * u[npne] + A9(au, npe, 9) * u[npnee];
        double sumve = A9(av, npe, 1) * v[nps] + A9(av, npe, 2) * v[npse] + A9(av, npe, 3) * v[npsee]
                     + A9(av, npe, 4) * v[np] + A9(av, npe, 6) * v[npee] + A9(av, npe, 7) * v[npn]
                     + A9(av, npe, 8) * v[npne] + A9(av, npe, 9) * v[npnee];
        double aux = (p[npn] + p[npne] - p[nps] - p[npse]) / 4.0;
        double pue = f.re[np] * (f.yke[np] * aux + f.ye[np] * (p[np] - p[npe]));
        double pve = f.re[np] * (-f.xke[np] * aux + f.xe[np] * (p[npe] - p[np]));
        double ue = ((mpa + mea) * f.uea[np] / dt + f.cup[np] + f.cup[npe] + f.sup[np] + f.sup[npe]
                     - sumup - sumue + 2.0 * pue) / (A9(au, np, 5) + A9(au, npe, 5));
        double ve = ((mpa + mea) * f.vea[np] / dt + f.cvp[np] + f.cvp[npe] + f.svp[np] + f.svp[npe]
                     - sumvp - sumve + 2.0 * pve) / (A9(av, np, 5) + A9(av, npe, 5));
        f.ue[np] = ue;
        f.ve[np] = ve;
        f.Uce[np] = ue * f.ye[np] - ve * f.xe[np];
    }
    if (j <= ny - 2) {
        const long long npnn = npn + nx, npnnw = npnn - 1, npnne = npnn + 1;
        const double mna = f.roa[npn] * f.rp[npn] / f.Jp[npn];
        double sumun = A9(au, npn, 1) * u[npw] + A9(au, npn, 2) * u[np] + A9(au, npn, 3) * u[npe]
                     + A9(au, npn, 4) * u[npnw] + A9(au, npn, 6) * u[npne] + A9(au, npn, 7) * u[npnnw]
                     + A9(au, npn, 8) * u[npnn] + A9(au, npn, 9) * u[npnne];
        double sumvn = A9(av, npn, 1) * v[npw] + A9(av, npn, 2) * v[np] + A9(av, npn, 3) * v[npe]
                     + A9(av, npn, 4) * v[npnw] + A9(av, npn, 6) * v[npne] + A9(av, npn, 7) * v[npnnw]
                     + A9(av, npn, 8) * v[npnn] + A9(av, npn, 9) * v[npnne];
        double aux = (p[npne] + p[npe] - p[npnw] - p[npw]) / 4.0;
        double pun = f.rn[np] * (f.yk[np] * (p[npn] - p[np]) - f.yen[np] * aux);
        double pvn = f.rn[np] * (f.xk[np] * (p[np] - p[npn]) + f.xen[np] * aux);
        double un = ((mpa + mna) * f.una[np] / dt + f.cup[np] + f.cup[npn] + f.sup[np] + f.sup[npn]
                     - sumup - sumun + 2.0 * pun) / (A9(au, np, 5) + A9(au, npn, 5));
        double vn = ((mpa + mna) * f.vna[np] / dt + f.cvp[np] + f.cvp[npn] + f.svp[np] + f.svp[npn]
                     - sumvp - sumvn + 2.0 * pvn) / (A9(av, np, 5) + A9(av, npn, 5));
        f.un[np] = un;
        f.vn[np] = vn;
        f.Vcn[np] = vn * f.xk[np] - un * f.yk[np];
    }
}
__global__ void k_faces_internal(Fields f, double dt, const double *dtp)
{
    CELL_IJ
    faces_internal_cell(f, dt, dtp, i, j);
}

__device__ __forceinline__ double sum9(const double *a, long long N, long long np)
{
    double s = 0.0;
#pragma unroll
    for (int k = 1; k <= 9; k++) s = s + A9(a, np, k);
    return s;
}

// get_internal_simplec_coefficients  src/equations/mach2d_coef.f90:1504-1600
__global__ void k_simplec_internal(Fields f)
{
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    CELL_IJ
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j);
    const double sau = sum9(f.au, N, np), sav = sum9(f.av, N, np);
    if (i <= nx - 2) {
        const long long npe = np + 1;
        double Lue = 2.0 * f.re[np] / (sau + sum9(f.au, N, npe));
        double Lve = 2.0 * f.re[np] / (sav + sum9(f.av, N, npe));
        double due = Lue * f.ye[np], dve = Lve * f.xe[np];
        f.due[np] = due; f.dve[np] = dve;
        f.de[np] = f.ye[np] * due + f.xe[np] * dve;
    }
    if (j <= ny - 2) {
        const long long npn = np + nx;
        double Lun = 2.0 * f.rn[np] / (sau + sum9(f.au, N, npn));
        double Lvn = 2.0 * f.rn[np] / (sav + sum9(f.av, N, npn));
        double dun = Lun * f.yk[np], dvn = Lvn * f.xk[np];
        f.dun[np] = dun; f.dvn[np] = dvn;
        f.dn[np] = f.xk[np] * dvn + f.yk[np] * dun;
    }
}

// get_pressure_correction_with_pl + get_density_correction_with_pl
// src/equations/mach2d_coef.f90:1602-1624
__global__ void k_p_ro_correction(Fields f, int do_p, int do_ro)
{
    long long N = (long long)f.nx * f.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N;
         k += (long long)gridDim.x * blockDim.x) {
        double pl = f.pl[k];
        if (do_p) f.p[k] = f.p[k] + pl;
        if (do_ro) f.ro[k] = f.ro[k] + pl * f.g[k];
    }
}

// get_u_v_at_real_nodes_with_pl  src/equations/mach2d_coef.f90:1626-1675
__global__ void k_uv_nodes_correction(Fields f)
{
    const int nx = f.nx, ny = f.ny;
    const long long N = (long long)nx * ny;
    CELL_IJ
    if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) return;
    const long long np = IDX(i, j), nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    const double *pl = f.pl, *xe = f.xe, *ye = f.ye, *xk = f.xk, *yk = f.yk;
    double plup = 0.5 * f.rp[np] * (+yk[np] * (pl[npn] + pl[np]) - yk[nps] * (pl[nps] + pl[np])
                                    - ye[np] * (pl[npe] + pl[np]) + ye[npw] * (pl[npw] + pl[np]));
    double plvp = 0.5 * f.rp[np] * (+xe[np] * (pl[np] + pl[npe]) - xe[npw] * (pl[np] + pl[npw])
                                    - xk[np] * (pl[np] + pl[npn]) + xk[nps] * (pl[np] + pl[nps]));
    f.u[np] = f.u[np] + plup / sum9(f.au, N, np);
    f.v[np] = f.v[np] + plvp / sum9(f.av, N, np);
}

// get_velocity_correction_at_faces_with_pl  src/equations/mach2d_coef.f90:1679-1758
__global__ void k_velocity_correction_faces(Fields f)
{
    const int nx = f.nx, ny = f.ny;
    CELL_IJ
    if (i > nx || j > ny) return;
    const long long np = IDX(i, j);
    const double *pl = f.pl;
    if (j >= 2 && j <= ny - 1 && i <= nx - 1) {
        const long long npe = np + 1;
        double ue = f.ue[np], ve = f.ve[np];
        f.Uce[np] = ue * f.ye[np] - ve * f.xe[np] + f.de[np] * (pl[np] - pl[npe]);
        f.ue[np] = ue + f.due[np] * (pl[np] - pl[npe]);
        f.ve[np] = ve + f.dve[np] * (pl[npe] - pl[np]);
    }
    if (j <= ny - 1 && i >= 2 && i <= nx - 1) {
        const long long npn = np + nx;
        double un = f.un[np], vn = f.vn[np];
        f.Vcn[np] = vn * f.xk[np] - un * f.yk[np] + f.dn[np] * (pl[np] - pl[npn]);
        f.un[np] = un + f.dun[np] * (pl[npn] - pl[np]);
        f.vn[np] = vn + f.dvn[np] * (pl[np] - pl[npn]);
    }
}

__device__ __forceinline__ void north_slip_inner(const Fields &f, int i, double &ub, double &vb);

// The p' cycle's update after the solve, fused: every face the reference's
// get_velocity_correction_at_faces_with_pl corrects (mach2d_coef.f90:
// 1679-1758) and intflow_velocities_at_boundary_faces then overwrites on the
// boundary (mod_intflow.f90:692-787) gets its final value directly (the
// boundary formula on the faces of columns 1 and nx-1 and rows 1 and ny-1,
// the correction elsewhere); then p += p', rho += g p' (:1602-1624); then
// max|p'| over all cells: block maxima combined with atomicMax on the bit
// patterns of non-negative doubles (order-independent, so deterministic).
// Each expression is the separate kernels', so the results are bitwise
// theirs.
__global__ void k_p_cycle_update(Fields f, int modvis, double *maxpl)
{
    const int nx = f.nx, ny = f.ny;
    CELL_IJ
    double m = 0.0;
    if (i <= nx && j <= ny) {
        const long long np = IDX(i, j);
        const double *pl = f.pl, *u = f.u, *v = f.v;
        if (j >= 2 && j <= ny - 1 && i <= nx - 1) {
            const long long npe = np + 1;
            if (i == 1) {
                const double ue = (u[np] + u[npe]) / 2.0, ve = 0.0;
                f.ue[np] = ue; f.ve[np] = ve;
                f.Uce[np] = ue * f.ye[np] - ve * f.xe[np];
            } else if (i == nx - 1) {
                const double ue = (u[np] + u[npe]) / 2.0, ve = (v[np] + v[npe]) / 2.0;
                f.ue[np] = ue; f.ve[np] = ve;
                f.Uce[np] = ue * f.ye[np] - ve * f.xe[np];
            } else {
                const double ue = f.ue[np], ve = f.ve[np];
                f.Uce[np] = ue * f.ye[np] - ve * f.xe[np] + f.de[np] * (pl[np] - pl[npe]);
                f.ue[np] = ue + f.due[np] * (pl[np] - pl[npe]);
                f.ve[np] = ve + f.dve[np] * (pl[npe] - pl[np]);
            }
        }
        if (j <= ny - 1 && i >= 2 && i <= nx - 1) {
            const long long npn = np + nx;
            if (j == 1) {
                f.un[np] = (u[np] + u[npn]) / 2.0;
                f.vn[np] = 0.0;
                f.Vcn[np] = 0.0;
            } else if (j == ny - 1) {
                double ub = 0.0, vb = 0.0;
                if (modvis == 0) north_slip_inner(f, i, ub, vb);
                f.un[np] = ub; f.vn[np] = vb; f.Vcn[np] = 0.0;
            } else {
                const double un = f.un[np], vn = f.vn[np];
                f.Vcn[np] = vn * f.xk[np] - un * f.yk[np] + f.dn[np] * (pl[np] - pl[npn]);
                f.un[np] = un + f.dun[np] * (pl[npn] - pl[np]);
                f.vn[np] = vn + f.dvn[np] * (pl[np] - pl[npn]);
            }
        }
        const double p1 = pl[np];
        f.p[np] = f.p[np] + p1;
        f.ro[np] = f.ro[np] + p1 * f.g[np];
        m = fmax(0.0, fabs(p1));
    }
    // block maximum, then one atomic per block
    __shared__ double wmax[8];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int w = threadIdx.y, lane = threadIdx.x;
    if (lane == 0) wmax[w] = m;
    __syncthreads();
    if (w == 0) {
        m = lane < 8 ? wmax[lane] : 0.0;
        for (int o = 4; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0 && maxpl)
            atomicMax(reinterpret_cast<unsigned long long *>(maxpl), (unsigned long long)__double_as_longlong(m));
    }
}

// initialize_boundary_faces_flags  src/equations/mach2d_coef.f90:1764-1828
__global__ void k_boundary_faces_flags(Fields f)
{
    const int nx = f.nx, ny = f.ny;
    CELL_IJ
    if (i > nx || j > ny) return;
    const long long np = IDX(i, j);
    f.fbe[np] = ((i == 1 || i == nx - 1) && j >= 2 && j <= ny - 1) ? 1.0 : 0.0;
    f.fbn[np] = ((j == 1 || j == ny - 1) && i >= 2 && i <= nx - 1) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------
// internal-flow boundary strips (src/user/internal_flow/mod_intflow.f90)

// get_u_v_north_slip, mod_intflow.f90:142-210: wall velocity for 2 <= i <= nx-1
__device__ __forceinline__ void north_slip_inner(const Fields &f, int i, double &ub, double &vb)
{
    const int nx = f.nx, ny = f.ny;
    const long long np = IDX(i, ny - 1);
    const double u = f.u[np], v = f.v[np], xk = f.xk[np], yk = f.yk[np];
    double Up = sqrt(u * u + v * v);
    double signal = copysign(1.0, xk * u + yk * v);
    double t = sqrt(xk * xk + yk * yk);
    double tx = xk / t, ty = yk / t;
    ub = signal * Up * tx;
    vb = signal * Up * ty;
}

// same routine for any 1 <= i <= nx, the two ends linearly extrapolated
__device__ void north_slip(const Fields &f, int i, double &ub, double &vb)
{
    const int nx = f.nx, ny = f.ny;
    if (i >= 2 && i <= nx - 1) { north_slip_inner(f, i, ub, vb); return; }
    double u2, v2, u3, v3;
    const double *x = f.x, *xp = f.xp;
    if (i == 1) {
        north_slip_inner(f, 2, u2, v2);
        north_slip_inner(f, 3, u3, v3);
        long long np = IDX(1, ny - 1), npe = np + 1, npee = npe + 1;
        ub = u2 + (u2 - u3) * (xp[npe] - x[np]) / (xp[npee] - xp[npe]);
        vb = v2 + (v2 - v3) * (xp[npe] - x[np]) / (xp[npee] - xp[npe]);
    } else {
        north_slip_inner(f, nx - 1, u2, v2);
        north_slip_inner(f, nx - 2, u3, v3);
        long long np = IDX(nx, ny - 1), npw = np - 1, npww = npw - 1;
        ub = u2 + (u2 - u3) * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]);
        vb = v2 + (v2 - v3) * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]);
    }
}

// boundary strip thread map: q in [0, 2*ny + 2*nx): west j, east j, south i, north i
__device__ __forceinline__ bool strip_of(int q, int nx, int ny, int &side, int &idx)
{
    if (q < ny) { side = 0; idx = q + 1; return true; }
    q -= ny;
    if (q < ny) { side = 1; idx = q + 1; return true; }
    q -= ny;
    if (q < nx) { side = 2; idx = q + 1; return true; }
    q -= nx;
    if (q < nx) { side = 3; idx = q + 1; return true; }
    return false;
}
#define STRIP_VARS                                              \
    const int nx = f.nx, ny = f.ny;                             \
    const long long N = (long long)nx * ny;                     \
    (void)N;
#define STRIP_HEAD                                              \
    const int nx = f.nx, ny = f.ny;                             \
    const long long N = (long long)nx * ny;                     \
    (void)N;                                                    \
    int side, idx;                                              \
    if (!strip_of(blockIdx.x * blockDim.x + threadIdx.x, nx, ny, side, idx)) return;

__device__ __forceinline__ void set_row9(double *a, long long N, long long np, int k1, double v1,
                                         int k2, double v2)
{
#pragma unroll
    for (int k = 1; k <= 9; k++) A9(a, np, k) = 0.0;
    A9(a, np, k1) = v1;
    A9(a, np, k2) = v2;
}

// intflow_set_bcu  mod_intflow.f90:214-301
__device__ __forceinline__ void set_bcu_strip(const Fields &f, int modvis, int side, int idx)
{
    STRIP_VARS
    const double *x = f.x, *xp = f.xp, *u = f.u;
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(1, j), npe = np + 1, npee = npe + 1;
        set_row9(f.au, N, np, 6, -1.0, 5, 1.0);
        f.bu[np] = (2.0 * xp[npe]) / (xp[npee] - xp[npe]) * (u[npe] - u[npee]);
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(nx, j), npw = np - 1, npww = npw - 1;
        set_row9(f.au, N, np, 4, -1.0, 5, 1.0);
        f.bu[np] = 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]) * (u[npw] - u[npww]);
    } else if (side == 2) {
        long long np = IDX(idx, 1);
        set_row9(f.au, N, np, 8, -1.0, 5, 1.0);
        f.bu[np] = 0.0;
    } else {
        long long np = IDX(idx, ny);
        set_row9(f.au, N, np, 2, 1.0, 5, 1.0);
        if (modvis == 1) f.bu[np] = 0.0;
        else { double ub, vb; north_slip(f, idx, ub, vb); f.bu[np] = 2.0 * ub; }
    }
}
__global__ void k_set_bcu(Fields f, int modvis)
{
    int side, idx;
    if (!strip_of(blockIdx.x * blockDim.x + threadIdx.x, f.nx, f.ny, side, idx)) return;
    set_bcu_strip(f, modvis, side, idx);
}

// intflow_set_bcv  mod_intflow.f90:305-392
__device__ __forceinline__ void set_bcv_strip(const Fields &f, int modvis, int side, int idx)
{
    STRIP_VARS
    const double *x = f.x, *xp = f.xp, *v = f.v;
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(1, j);
        set_row9(f.av, N, np, 6, 1.0, 5, 1.0);
        f.bv[np] = 0.0;
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(nx, j), npw = np - 1, npww = npw - 1;
        set_row9(f.av, N, np, 4, -1.0, 5, 1.0);
        f.bv[np] = (v[npw] - v[npww]) * 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]);
    } else if (side == 2) {
        long long np = IDX(idx, 1);
        set_row9(f.av, N, np, 8, 1.0, 5, 1.0);
        f.bv[np] = 0.0;
    } else {
        long long np = IDX(idx, ny);
        set_row9(f.av, N, np, 2, 1.0, 5, 1.0);
        if (modvis == 1) f.bv[np] = 0.0;
        else { double ub, vb; north_slip(f, idx, ub, vb); f.bv[np] = 2.0 * vb; }
    }
}
__global__ void k_set_bcv(Fields f, int modvis)
{
    int side, idx;
    if (!strip_of(blockIdx.x * blockDim.x + threadIdx.x, f.nx, f.ny, side, idx)) return;
    set_bcv_strip(f, modvis, side, idx);
}

__device__ __forceinline__ void set_row5(double *a, long long N, long long np, int k1, double v1)
{
#pragma unroll
    for (int k = 1; k <= 5; k++) A9(a, np, k) = 0.0;
    A9(a, np, k1) = v1;
    A9(a, np, 3) = 1.0;
}

// intflow_set_bcpl  mod_intflow.f90:396-459 (corner rows untouched)
__device__ __forceinline__ void set_bcpl_strip(const Fields &f, int side, int idx)
{
    STRIP_VARS
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(1, j);
        set_row5(f.ap, N, np, 4, 1.0);
        f.bp[np] = 2.0 * f.plin[j - 1];
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(nx, j), npw = np - 1, npww = npw - 1;
        set_row5(f.ap, N, np, 2, -1.0);
        f.bp[np] = 2.0 * (f.x[npw] - f.xp[npw]) / (f.xp[npw] - f.xp[npww]) * (f.pl[npw] - f.pl[npww]);
    } else if (side == 2) {
        if (idx < 2 || idx > nx - 1) return;
        long long np = IDX(idx, 1);
        set_row5(f.ap, N, np, 5, -1.0);
        f.bp[np] = 0.0;
    } else {
        if (idx < 2 || idx > nx - 1) return;
        long long np = IDX(idx, ny);
        set_row5(f.ap, N, np, 1, -1.0);
        f.bp[np] = 0.0;
    }
}
__global__ void k_set_bcpl(Fields f)
{
    int side, idx;
    if (!strip_of(blockIdx.x * blockDim.x + threadIdx.x, f.nx, f.ny, side, idx)) return;
    set_bcpl_strip(f, side, idx);
}

// intflow_set_bcT  mod_intflow.f90:464-550
__global__ void k_set_bcT(Fields f, double Twall)
{
    STRIP_HEAD
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(1, j);
        set_row9(f.at, N, np, 6, 1.0, 5, 1.0);
        f.bt[np] = 2.0 * f.Tin[j - 1];
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(nx, j), npw = np - 1, npww = npw - 1;
        set_row9(f.at, N, np, 4, -1.0, 5, 1.0);
        f.bt[np] = 2.0 * (f.x[npw] - f.xp[npw]) / (f.xp[npw] - f.xp[npww]) * (f.T[npw] - f.T[npww]);
    } else if (side == 2) {
        long long np = IDX(idx, 1);
        set_row9(f.at, N, np, 8, -1.0, 5, 1.0);
        f.bt[np] = 0.0;
    } else {
        long long np = IDX(idx, ny);
        if (Twall > 0.0) { set_row9(f.at, N, np, 2, 1.0, 5, 1.0); f.bt[np] = 2.0 * Twall; }
        else { set_row9(f.at, N, np, 2, -1.0, 5, 1.0); f.bt[np] = 0.0; }
    }
}

// intflow_velocities_at_boundary_faces  mod_intflow.f90:692-787
__device__ __forceinline__ void faces_boundary_strip(const Fields &f, int modvis, int side, int idx)
{
    STRIP_VARS
    const double *u = f.u, *v = f.v;
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(1, j), npe = np + 1;
        double ue = (u[np] + u[npe]) / 2.0, ve = 0.0;
        f.ue[np] = ue; f.ve[np] = ve;
        f.Uce[np] = ue * f.ye[np] - ve * f.xe[np];
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(nx - 1, j), npe = np + 1;
        double ue = (u[np] + u[npe]) / 2.0, ve = (v[np] + v[npe]) / 2.0;
        f.ue[np] = ue; f.ve[np] = ve;
        f.Uce[np] = ue * f.ye[np] - ve * f.xe[np];
    } else if (side == 2) {
        int i = idx; if (i < 2 || i > nx - 1) return;
        long long np = IDX(i, 1), npn = np + nx;
        f.un[np] = (u[np] + u[npn]) / 2.0;
        f.vn[np] = 0.0;
        f.Vcn[np] = 0.0;
    } else {
        int i = idx; if (i < 2 || i > nx - 1) return;
        long long np = IDX(i, ny - 1);
        double ub = 0.0, vb = 0.0;
        if (modvis == 0) north_slip_inner(f, i, ub, vb);
        f.un[np] = ub; f.vn[np] = vb; f.Vcn[np] = 0.0;
    }
}
__global__ void k_faces_boundary(Fields f, int modvis)
{
    int side, idx;
    if (!strip_of(blockIdx.x * blockDim.x + threadIdx.x, f.nx, f.ny, side, idx)) return;
    faces_boundary_strip(f, modvis, side, idx);
}

// intflow_boundary_simplec  mod_intflow.f90:791-877
__global__ void k_boundary_simplec(Fields f)
{
    STRIP_HEAD
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(1, j);
        f.due[np] = f.due[np + 1]; f.dve[np] = 0.0; f.de[np] = f.de[np + 1];
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        long long np = IDX(nx - 1, j);
        f.due[np] = f.due[np - 1]; f.dve[np] = f.dve[np - 1]; f.de[np] = f.de[np - 1];
    } else if (side == 2) {
        int i = idx; if (i < 2 || i > nx - 1) return;
        long long np = IDX(i, 1);
        f.dun[np] = f.dun[np + nx]; f.dvn[np] = 0.0; f.dn[np] = 0.0;
    } else {
        int i = idx; if (i < 2 || i > nx - 1) return;
        long long np = IDX(i, ny - 1);
        f.dun[np] = 0.0; f.dvn[np] = 0.0; f.dn[np] = 0.0;
    }
}

// ghost values of intflow_extrapolate_u_v_to_fictitious (mod_intflow.f90:881-964)
__device__ __forceinline__ void west_ghost_uv(const Fields &f, int j, double &uo, double &vo)
{
    const int nx = f.nx;
    long long np = IDX(1, j), npe = np + 1, npee = np + 2;
    const double *u = f.u, *xp = f.xp;
    uo = u[npe] + 2.0 * xp[npe] / (xp[npee] - xp[npe]) * (u[npe] - u[npee]);
    vo = -f.v[npe];
}
__device__ __forceinline__ void east_ghost_uv(const Fields &f, int j, double &uo, double &vo)
{
    const int nx = f.nx;
    long long np = IDX(nx, j), npw = np - 1, npww = np - 2;
    const double *u = f.u, *v = f.v, *x = f.x, *xp = f.xp;
    uo = u[npw] + 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]) * (u[npw] - u[npww]);
    vo = v[npw] + 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]) * (v[npw] - v[npww]);
}

__global__ void k_extrapolate_uv(Fields f, int modvis)
{
    STRIP_HEAD
    double uo, vo;
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        west_ghost_uv(f, j, uo, vo);
        long long np = IDX(1, j); f.u[np] = uo; f.v[np] = vo;
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        east_ghost_uv(f, j, uo, vo);
        long long np = IDX(nx, j); f.u[np] = uo; f.v[np] = vo;
    } else if (side == 2) {
        // south row: u(i,1) = u(i,2), v(i,1) = -v(i,2); the corners read the
        // west/east ghosts of row 2 that this routine has just updated
        int i = idx;
        double un, vn;
        if (i == 1) west_ghost_uv(f, 2, un, vn);
        else if (i == nx) east_ghost_uv(f, 2, un, vn);
        else { un = f.u[IDX(i, 2)]; vn = f.v[IDX(i, 2)]; }
        long long np = IDX(i, 1); f.u[np] = un; f.v[np] = -vn;
    } else {
        int i = idx;
        double us, vs;
        if (i == 1) west_ghost_uv(f, ny - 1, us, vs);
        else if (i == nx) east_ghost_uv(f, ny - 1, us, vs);
        else { us = f.u[IDX(i, ny - 1)]; vs = f.v[IDX(i, ny - 1)]; }
        long long np = IDX(i, ny);
        if (modvis == 1) { f.u[np] = -us; f.v[np] = -vs; }
        else {
            double ub, vb; north_slip(f, i, ub, vb);
            f.u[np] = -us + 2.0 * ub; f.v[np] = -vs + 2.0 * vb;
        }
    }
}

// T = (Href - (u^2+v^2)/2)/Cpref  src/mach2d_main.f90:362
__global__ void k_T_from_H_nodes(Fields f, double Href, double Cpref)
{
    long long N = (long long)f.nx * f.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N;
         k += (long long)gridDim.x * blockDim.x)
        f.T[k] = (Href - (f.u[k] * f.u[k] + f.v[k] * f.v[k]) / 2.0) / Cpref;
}

// intflow_boundary_T_from_H_conservation  mod_intflow.f90:557-688
__device__ __forceinline__ double east_T_ghost(const Fields &f, int j, double Href, double Cpref, double *Tbe)
{
    const int nx = f.nx;
    long long np = IDX(nx - 1, j);
    double tb = (Href - (f.ue[np] * f.ue[np] + f.ve[np] * f.ve[np]) / 2.0) / Cpref;
    if (Tbe) Tbe[j - 1] = tb;
    return 2.0 * tb - f.T[np];
}
__device__ __forceinline__ double west_T_ghost(const Fields &f, int j, double *Tbw)
{
    const int nx = f.nx;
    long long np = IDX(1, j);
    double tb = f.Tin[j - 1];
    if (Tbw) Tbw[j - 1] = tb;
    return 2.0 * tb - f.T[np + 1];
}
__global__ void k_T_boundary_H(Fields f, double Href, double Cpref)
{
    STRIP_HEAD
    if (side == 0) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        f.T[IDX(1, j)] = west_T_ghost(f, j, f.Tbw);
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        f.T[IDX(nx, j)] = east_T_ghost(f, j, Href, Cpref, f.Tbe);
    } else if (side == 3) {
        int i = idx;
        if (i >= 2 && i <= nx - 1) {
            long long np = IDX(i, ny - 1);
            double tb = (Href - (f.un[np] * f.un[np] + f.vn[np] * f.vn[np]) / 2.0) / Cpref;
            f.Tbn[i - 1] = tb;
            f.T[np + nx] = 2.0 * tb - f.T[np];
        } else if (i == 1) {
            f.T[IDX(1, ny)] = west_T_ghost(f, ny - 1, nullptr);
        } else {
            f.T[IDX(nx, ny)] = east_T_ghost(f, ny - 1, Href, Cpref, nullptr);
        }
    } else {
        int i = idx;
        if (i >= 2 && i <= nx - 1) {
            long long np = IDX(i, 1);
            double tb = (Href - (f.un[np] * f.un[np] + f.vn[np] * f.vn[np]) / 2.0) / Cpref;
            f.Tbs[i - 1] = tb;
            f.T[np] = 2.0 * tb - f.T[np + nx];
        } else if (i == 1) {
            f.T[IDX(1, 1)] = west_T_ghost(f, 2, nullptr);
        } else {
            f.T[IDX(nx, 1)] = east_T_ghost(f, 2, Href, Cpref, nullptr);
        }
    }
}

// intflow_time_cycle_update  mod_intflow.f90:1106-1134
//   (get_uin_vin_pin_Tin_Mw :968-1006, get_plin_and_p_fictitious :1010-1101)
__device__ __forceinline__ double inlet_pin(const Fields &f, const Params &q, int j, bool store)
{
    const int nx = f.nx;
    long long np = IDX(1, j), npe = np + 1;
    double uin = (f.u[np] + f.u[npe]) / 2.0, vin = 0.0;
    double gamma = q.gamma, Rg = q.Rg;
    double Tin = q.T0 - (gamma - 1.0) / (2.0 * gamma * Rg) * (uin * uin + vin * vin);
    double Mw = sqrt((uin * uin + vin * vin) / (gamma * Rg * Tin));
    double pin = q.p0 * pow(1.0 + 0.5 * (gamma - 1.0) * (Mw * Mw), -gamma / (gamma - 1.0));
    if (store) {
        f.pina[j - 1] = f.pin[j - 1];
        f.uin[j - 1] = uin; f.vin[j - 1] = vin; f.Tin[j - 1] = Tin; f.Mw[j - 1] = Mw;
        f.plin[j - 1] = pin - f.pin[j - 1];
        f.pin[j - 1] = pin;
    }
    return pin;
}
__device__ __forceinline__ double east_p_ghost(const Fields &f, int j)
{
    const int nx = f.nx;
    long long np = IDX(nx, j), npw = np - 1, npww = npw - 1;
    const double *p = f.p, *x = f.x, *xp = f.xp;
    return p[npw] + 2.0 * (x[npw] - xp[npw]) / (xp[npw] - xp[npww]) * (p[npw] - p[npww]);
}
__global__ void k_inlet_update(Fields f, Params q)
{
    STRIP_HEAD
    if (side == 0) {
        int j = idx;
        if (j < 2 || j > ny - 1) { f.pina[j - 1] = f.pin[j - 1]; return; }   // pina = pin, whole array
        // new inlet state of row j (only this thread touches pin(j)); the
        // corner threads recompute the same value without storing it
        long long np = IDX(1, j);
        double pnew = inlet_pin(f, q, j, true);
        f.p[np] = 2.0 * pnew - f.p[np + 1];
    } else if (side == 1) {
        int j = idx; if (j < 2 || j > ny - 1) return;
        f.p[IDX(nx, j)] = east_p_ghost(f, j);
    } else if (side == 2) {
        int i = idx;
        double pv;
        if (i == 1) pv = 2.0 * inlet_pin(f, q, 2, false) - f.p[IDX(2, 2)];
        else if (i == nx) pv = east_p_ghost(f, 2);
        else pv = f.p[IDX(i, 2)];
        f.p[IDX(i, 1)] = pv;
    } else {
        int i = idx;
        double pv;
        if (i == 1) pv = 2.0 * inlet_pin(f, q, ny - 1, false) - f.p[IDX(2, ny - 1)];
        else if (i == nx) pv = east_p_ghost(f, ny - 1);
        else pv = f.p[IDX(i, ny - 1)];
        f.p[IDX(i, ny)] = pv;
    }
}

// g = 1/(Rg T)  src/mach2d_main.f90:156
__global__ void k_g(Fields f, double Rg)
{
    long long N = (long long)f.nx * f.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N;
         k += (long long)gridDim.x * blockDim.x)
        f.g[k] = 1.0 / (Rg * f.T[k]);
}

// previous time level  src/mach2d_main.f90:96-104
__global__ void k_backup(Fields f)
{
    long long N = (long long)f.nx * f.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N;
         k += (long long)gridDim.x * blockDim.x) {
        // all nine loads before any store: the planes are distinct, and loads
        // in flight together keep the copy bandwidth-bound
        const double ro = __ldg(f.ro + k), T = __ldg(f.T + k), p = __ldg(f.p + k), u = __ldg(f.u + k);
        const double v = __ldg(f.v + k), ue = __ldg(f.ue + k), ve = __ldg(f.ve + k), un = __ldg(f.un + k);
        const double vn = __ldg(f.vn + k);
        f.roa[k] = ro; f.Ta[k] = T; f.pa[k] = p; f.ua[k] = u; f.va[k] = v;
        f.uea[k] = ue; f.vea[k] = ve; f.una[k] = un; f.vna[k] = vn;
    }
}

// ---- fused launches: kernels whose cells are disjoint and that read none of
// each other's outputs run as one launch, every cell computed by the same
// device function as in its own kernel (bitwise the separate launches)

// ring cell (i, j) -> the strip entry of the boundary kernels that covers it
// (the corners belong to the south and north strips; the west and east
// strips skip them)
__device__ __forceinline__ bool ring_strip(int i, int j, int nx, int ny, int &side, int &idx)
{
    if (j == 1) { side = 2; idx = i; return true; }
    if (j == ny) { side = 3; idx = i; return true; }
    if (i == 1) { side = 0; idx = j; return true; }
    if (i == nx) { side = 1; idx = j; return true; }
    return false;
}

// u and v coefficients and sources on the real cells, intflow_set_bcu/bcv on
// the ring
__global__ void k_uv_assembly_bc(Fields f, Params q, int modvis)
{
    CELL_IJ
    if (i > f.nx || j > f.ny) return;
    int side, idx;
    if (ring_strip(i, j, f.nx, f.ny, side, idx)) {
        set_bcu_strip(f, modvis, side, idx);
        set_bcv_strip(f, modvis, side, idx);
    } else {
        u_assembly_cell(f, q, ASM_COEF | ASM_SRC, i, j);
        v_assembly_cell(f, q, ASM_COEF | ASM_SRC, i, j);
    }
}

// the internal face velocities and the boundary faces
__global__ void k_faces_all(Fields f, double dt, const double *dtp, int modvis)
{
    CELL_IJ
    if (i > f.nx || j > f.ny) return;
    int side, idx;
    if (ring_strip(i, j, f.nx, f.ny, side, idx)) faces_boundary_strip(f, modvis, side, idx);
    else faces_internal_cell(f, dt, dtp, i, j);
}

// the p' coefficients and source of one cycle and intflow_set_bcpl
__global__ void k_p_assembly_bc(Fields f, Params q)
{
    CELL_IJ
    if (i > f.nx || j > f.ny) return;
    int side, idx;
    if (ring_strip(i, j, f.nx, f.ny, side, idx)) {
        if (i == 1 && j == 1 && q.maxpl) *q.maxpl = 0.0;   // as p_assembly_cell does at (1, 1)
        set_bcpl_strip(f, side, idx);
    } else {
        p_assembly_cell(f, q, ASM_COEF | ASM_SRC, i, j);
    }
}

// ---------------------------------------------------------------------------
static inline dim3 grid1d(long long N)
{
    long long b = (N + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return dim3((unsigned)b);
}
static inline dim3 grid_strip(int nx, int ny)
{
    return dim3((unsigned)((2 * nx + 2 * ny + 127) / 128));
}

cudaError_t launch_uv_assembly_bc(const Fields &f, const Params &q, int modvis, cudaStream_t st)
{ k_uv_assembly_bc<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, q, modvis); return cudaGetLastError(); }
cudaError_t launch_faces_all(const Fields &f, double dt, int modvis, cudaStream_t st, const double *dtp)
{ k_faces_all<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, dt, dtp, modvis); return cudaGetLastError(); }
cudaError_t launch_p_assembly_bc(const Fields &f, const Params &q, cudaStream_t st)
{ k_p_assembly_bc<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, q); return cudaGetLastError(); }
cudaError_t launch_density_at_nodes(const Fields &f, double Rg, cudaStream_t st)
{ k_density_nodes<<<grid1d((long long)f.nx * f.ny), 256, 0, st>>>(f, Rg); return cudaGetLastError(); }
cudaError_t launch_density_at_faces(const Fields &f, double beta, cudaStream_t st)
{ k_density_faces<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, beta); return cudaGetLastError(); }
cudaError_t launch_u_assembly(const Fields &f, const Params &q, int what, cudaStream_t st)
{ k_u_assembly<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, q, what); return cudaGetLastError(); }
cudaError_t launch_v_assembly(const Fields &f, const Params &q, int what, cudaStream_t st)
{ k_v_assembly<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, q, what); return cudaGetLastError(); }
cudaError_t launch_T_assembly(const Fields &f, const Params &q, cudaStream_t st)
{ k_T_assembly<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, q); return cudaGetLastError(); }
cudaError_t launch_p_assembly(const Fields &f, const Params &q, int what, cudaStream_t st)
{ k_p_assembly<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, q, what); return cudaGetLastError(); }
cudaError_t launch_velocities_at_internal_faces(const Fields &f, double dt, cudaStream_t st, const double *dtp)
{ k_faces_internal<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, dt, dtp); return cudaGetLastError(); }
cudaError_t launch_internal_simplec(const Fields &f, cudaStream_t st)
{ k_simplec_internal<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f); return cudaGetLastError(); }
cudaError_t launch_p_ro_correction(const Fields &f, int do_p, int do_ro, cudaStream_t st)
{ k_p_ro_correction<<<grid1d((long long)f.nx * f.ny), 256, 0, st>>>(f, do_p, do_ro); return cudaGetLastError(); }
cudaError_t launch_uv_nodes_correction(const Fields &f, cudaStream_t st)
{ k_uv_nodes_correction<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f); return cudaGetLastError(); }
cudaError_t launch_velocity_correction_at_faces(const Fields &f, cudaStream_t st)
{ k_velocity_correction_faces<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f); return cudaGetLastError(); }
cudaError_t launch_p_cycle_update(const Fields &f, int modvis, double *maxpl, cudaStream_t st)
{ k_p_cycle_update<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, modvis, maxpl); return cudaGetLastError(); }
cudaError_t launch_boundary_faces_flags(const Fields &f, cudaStream_t st)
{ k_boundary_faces_flags<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f); return cudaGetLastError(); }
cudaError_t launch_set_bcu(const Fields &f, int modvis, cudaStream_t st)
{ k_set_bcu<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, modvis); return cudaGetLastError(); }
cudaError_t launch_set_bcv(const Fields &f, int modvis, cudaStream_t st)
{ k_set_bcv<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, modvis); return cudaGetLastError(); }
cudaError_t launch_set_bcpl(const Fields &f, cudaStream_t st)
{ k_set_bcpl<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f); return cudaGetLastError(); }
cudaError_t launch_set_bcT(const Fields &f, double Twall, cudaStream_t st)
{ k_set_bcT<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, Twall); return cudaGetLastError(); }
cudaError_t launch_velocities_at_boundary_faces(const Fields &f, int modvis, cudaStream_t st)
{ k_faces_boundary<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, modvis); return cudaGetLastError(); }
cudaError_t launch_boundary_simplec(const Fields &f, cudaStream_t st)
{ k_boundary_simplec<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f); return cudaGetLastError(); }
cudaError_t launch_extrapolate_uv(const Fields &f, int modvis, cudaStream_t st)
{ k_extrapolate_uv<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, modvis); return cudaGetLastError(); }
cudaError_t launch_T_from_H(const Fields &f, double Href, double Cpref, cudaStream_t st)
{
    k_T_from_H_nodes<<<grid1d((long long)f.nx * f.ny), 256, 0, st>>>(f, Href, Cpref);
    k_T_boundary_H<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, Href, Cpref);
    return cudaGetLastError();
}
cudaError_t launch_T_boundary_H(const Fields &f, double Href, double Cpref, cudaStream_t st)
{ k_T_boundary_H<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, Href, Cpref); return cudaGetLastError(); }
cudaError_t launch_inlet_update(const Fields &f, const Params &q, cudaStream_t st)
{ k_inlet_update<<<grid_strip(f.nx, f.ny), 128, 0, st>>>(f, q); return cudaGetLastError(); }
cudaError_t launch_g(const Fields &f, double Rg, cudaStream_t st)
{ k_g<<<grid1d((long long)f.nx * f.ny), 256, 0, st>>>(f, Rg); return cudaGetLastError(); }
cudaError_t launch_backup(const Fields &f, cudaStream_t st)
{ k_backup<<<grid1d((long long)f.nx * f.ny), 256, 0, st>>>(f); return cudaGetLastError(); }

}  // namespace m2d
