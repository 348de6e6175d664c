// m2d_setup.h -- host-side part of the instance set-up (grid nodes and the
// strips of the initial guess).
#pragma once
#include <utility>
#include <vector>
#include "../../include/mach2d_b200.h"

namespace m2d {

// X-macro of the N-sized planes that one instance keeps on the device,
// named as the reference's module variables (src/mod_mach2d_data.f90:30-173)
#define M2D_PLANES(X)                                                          \
    X(x) X(y) X(xp) X(yp) X(xe) X(ye) X(xen) X(yen) X(xk) X(yk) X(xke) X(yke)  \
    X(Jp) X(Je) X(Jn) X(alphae) X(gamman) X(betae) X(betan) X(radius) X(re)    \
    X(rn) X(rp) X(fbe) X(fbn) X(p) X(pa) X(T) X(Ta) X(ro) X(roa) X(roe) X(ron) \
    X(g) X(u) X(ua) X(v) X(va) X(ue) X(un) X(ve) X(vn) X(Uce) X(Vcn) X(uea)    \
    X(vea) X(una) X(vna) X(cp) X(vlp) X(vle) X(vln) X(kp) X(ke) X(kn) X(cup)   \
    X(sup) X(cvp) X(svp) X(bu) X(bv) X(bt) X(bp) X(pl) X(due) X(dve) X(dun)    \
    X(dvn) X(de) X(dn) X(vtp)

// what the host computes of one instance: the grid nodes and the strips of
// the initial guess; everything else is computed on the device
struct HostInstance {
    int nx = 0, ny = 0;
    std::vector<double> x, y;                                 // N: grid nodes
    std::vector<double> M1D, p1D, T1D, u1D;                   // nx: quasi-1D isentropic flow
    std::vector<double> ue1D;                                 // nx: isentropic east-face u of column i
    std::vector<double> col;                                  // 4 nx: p1D, T1D, u1D, ue1D of the columns
    std::vector<double> uin, vin, pin, Tin, Mw;               // ny: inlet strips
    std::vector<double> Tbe, Tbw, Tbn, Tbs;                   // ny, ny, nx, nx
    double Sg = 0, fm1D = 0, Fd1D = 0, Fpv1D = 0, Rg = 0, gamma = 0, Cpref = 0, Href = 0, dt0 = 0;
};

// the grid nodes, reference values and the column strips; returns 0 or an
// M2D_ERR_* code
int build_instance(const m2d_case &c, HostInstance &h);
// the inlet strips (get_uin_vin_pin_Tin_Mw, mod_intflow.f90:968-1000) from
// uin(j) = (u(1,j) + u(2,j)) / 2 of the extrapolated initial field, and Tbw
void inlet_strips(const m2d_case &c, HostInstance &h, const std::vector<double> &uin);
double mach_area(int kf, double ar, double gamma);
double ramp_dt(int it, const m2d_case &c);

}  // namespace m2d
