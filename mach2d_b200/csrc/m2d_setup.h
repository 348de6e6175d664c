// m2d_setup.h -- host-side instance set-up (grid, metrics, initial guess).
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
    X(dvn) X(de) X(dn)

struct HostInstance {
    int nx = 0, ny = 0;
#define M2D_DECL_VEC(name) std::vector<double> name;
    M2D_PLANES(M2D_DECL_VEC)
#undef M2D_DECL_VEC
    std::vector<double> uin, vin, pin, Tin, Mw, plin, pina;   // ny
    std::vector<double> Tbe, Tbw, Tbn, Tbs;                   // ny, ny, nx, nx
    std::vector<double> M1D, p1D, T1D, u1D;                   // nx
    double Sg = 0, fm1D = 0, Fd1D = 0, Fpv1D = 0, Rg = 0, gamma = 0, Cpref = 0, Href = 0, dt0 = 0;

    std::vector<std::pair<const char *, std::vector<double> *>> planes()
    {
        std::vector<std::pair<const char *, std::vector<double> *>> lst_;
#define M2D_LIST_VEC(name) lst_.push_back({#name, &this->name});
        M2D_PLANES(M2D_LIST_VEC)
#undef M2D_LIST_VEC
        return lst_;
    }
};

// builds the grid, metrics and initial fields; returns 0 or an M2D_ERR_* code
int build_instance(const m2d_case &c, HostInstance &h);
double mach_area(int kf, double ar, double gamma);
double ramp_dt(int it, const m2d_case &c);
void north_slip_host(int nx, int ny, const std::vector<double> &x, const std::vector<double> &xp,
                     const std::vector<double> &xk, const std::vector<double> &yk,
                     const std::vector<double> &u, const std::vector<double> &v,
                     std::vector<double> &ubn, std::vector<double> &vbn);

}  // namespace m2d
