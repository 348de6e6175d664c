"""The routines of `module coefficients` (src/equations/mach2d_coef.f90) and
of the internal-flow plug-in (src/user/internal_flow/mod_intflow.f90), with
the reference's argument lists and order.

Arrays are float64 numpy arrays in the reference layout (a(nx*ny, k) as a
(k, nx*ny) array); arguments the reference declares intent(out) or
intent(inout) are updated in place.  Scalars are Python numbers.  Each call
runs the corresponding CUDA kernel through the C ABI.
"""
import ctypes

from ._lib import call

_INT = {"nx", "ny", "modvis", "coord"}
_DBL = {"dt", "beta", "Rg", "Twall", "Cpref", "Href", "gamma", "P0", "T0"}


def _make(name, params, doc, out_scalar=None):
    cname = "m2d_" + name

    def fn(*args):
        if len(args) != len(params):
            raise TypeError(f"{name} takes {len(params)} arguments ({len(args)} given)")
        conv = []
        for p, a in zip(params, args):
            if p in _INT:
                conv.append(int(a))
            elif p in _DBL:
                conv.append(float(a))
            else:
                conv.append(a)
        if out_scalar:
            res = ctypes.c_double(0.0)
            call(cname, *conv, res)
            return res.value
        call(cname, *conv)

    fn.__name__ = name
    fn.__doc__ = doc
    return fn


def _p(s):
    return [t.strip() for t in s.split(",")]


get_density_at_nodes = _make("get_density_at_nodes", _p("nx, ny, Rg, p, T, ro"), "mach2d_coef.f90:6-17")
get_density_at_faces = _make("get_density_at_faces", _p("nx, ny, beta, ro, Uce, Vcn, roe, ron"),
                             "mach2d_coef.f90:20-60")
get_u_coefficients = _make("get_u_coefficients", _p(
    "nx, ny, modvis, dt, rp, re, rn, Jp, Je, Jn, ye, yk, alphae, betae, betan, gamman, "
    "vle, vln, roe, ron, roa, Uce, Vcn, a"), "mach2d_coef.f90:63-218")
get_u_source = _make("get_u_source", _p(
    "nx, ny, modvis, beta, dt, rp, re, rn, xe, ye, xk, yk, xke, yke, xen, yen, Jp, Je, Jn, "
    "roe, ron, roa, p, vle, vln, Uce, Vcn, ua, u, v, cup, sup, b"), "mach2d_coef.f90:221-451")
get_v_coefficients = _make("get_v_coefficients", _p(
    "nx, ny, coord, modvis, dt, rp, re, rn, Jp, Je, Jn, xe, xk, alphae, betae, betan, gamman, "
    "vle, vln, vlp, roe, ron, roa, Uce, Vcn, a"), "mach2d_coef.f90:454-613")
get_v_source = _make("get_v_source", _p(
    "nx, ny, coord, modvis, beta, dt, rp, re, rn, xe, ye, xk, yk, xke, yke, xen, yen, Jp, Je, "
    "Jn, roe, ron, roa, p, vle, vln, Uce, Vcn, va, u, v, cvp, svp, b"), "mach2d_coef.f90:616-783")
get_T_coefficients_and_source = _make("get_T_coefficients_and_source", _p(
    "nx, ny, modvis, beta, dt, rp, re, rn, xe, ye, xk, yk, xke, yke, xen, yen, alphae, betae, "
    "betan, gamman, Jp, Je, Jn, roe, ron, ro, roa, p, pa, cp, vle, vln, ke, kn, Uce, Vcn, u, v, "
    "ue, ve, un, vn, ua, va, T, Ta, fbe, fbn, a, b"), "mach2d_coef.f90:787-1203")
get_p_coefficients = _make("get_p_coefficients", _p(
    "nx, ny, dt, rp, re, rn, Jp, Uce, Vcn, roe, ron, g, de, dn, a"), "mach2d_coef.f90:1207-1278")
get_p_source = _make("get_p_source", _p(
    "nx, ny, dt, rp, re, rn, Jp, roe, ron, ro, roa, Uce, Vcn, de, dn, g, pl, b"),
    "mach2d_coef.f90:1281-1348")
get_velocities_at_internal_faces = _make("get_velocities_at_internal_faces", _p(
    "nx, ny, dt, rp, re, rn, xe, ye, xk, yk, xen, yen, xke, yke, Jp, cup, cvp, sup, svp, au, av, "
    "roa, p, u, v, uea, vea, una, vna, ue, ve, un, vn, Uce, Vcn"), "mach2d_coef.f90:1350-1501")
get_internal_simplec_coefficients = _make("get_internal_simplec_coefficients", _p(
    "nx, ny, re, rn, xe, ye, xk, yk, au, av, due, dve, dun, dvn, de, dn"), "mach2d_coef.f90:1504-1600")
get_pressure_correction_with_pl = _make("get_pressure_correction_with_pl", _p("nx, ny, pl, p"),
                                        "mach2d_coef.f90:1602-1611")
get_density_correction_with_pl = _make("get_density_correction_with_pl", _p("nx, ny, pl, g, ro"),
                                       "mach2d_coef.f90:1614-1624")
get_u_v_at_real_nodes_with_pl = _make("get_u_v_at_real_nodes_with_pl", _p(
    "nx, ny, xe, ye, xk, yk, rp, pl, au, av, u, v"), "mach2d_coef.f90:1626-1675")
get_velocity_correction_at_faces_with_pl = _make("get_velocity_correction_at_faces_with_pl", _p(
    "nx, ny, xe, ye, xk, yk, due, dve, dun, dvn, de, dn, pl, ue, ve, un, vn, Uce, Vcn"),
    "mach2d_coef.f90:1679-1758")
initialize_boundary_faces_flags = _make("initialize_boundary_faces_flags", _p("nx, ny, fbe, fbn"),
                                        "mach2d_coef.f90:1764-1828")
check_mass_conservation = _make("check_mass_conservation", _p(
    "nx, ny, dt, rp, re, rn, Jp, ro, roa, ron, roe, Uce, Vcn"), "mach2d_coef.f90:1833-1880 (returns res)",
    out_scalar=True)

# internal-flow plug-in (derived-type members passed as plain arrays/scalars)
intflow_set_bcu = _make("intflow_set_bcu", _p("nx, ny, modvis, x, xp, xk, yk, u, v, au, b"),
                        "mod_intflow.f90:214-301")
intflow_set_bcv = _make("intflow_set_bcv", _p("nx, ny, modvis, x, xp, xk, yk, u, v, av, b"),
                        "mod_intflow.f90:305-392")
intflow_set_bcpl = _make("intflow_set_bcpl", _p("nx, ny, x, xp, pl, plin, ap, bp"),
                         "mod_intflow.f90:396-459 (plin = iflow%plin)")
intflow_set_bcT = _make("intflow_set_bcT", _p("nx, ny, x, xp, T, Twall, Tin, at, bt"),
                        "mod_intflow.f90:464-550 (Twall, Tin = iflow%Twall, iflow%Tin)")
intflow_boundary_T_from_H_conservation = _make("intflow_boundary_T_from_H_conservation", _p(
    "nx, ny, Cpref, Href, Tin, u, ue, un, v, ve, vn, T, Tbe, Tbw, Tbn, Tbs"), "mod_intflow.f90:557-688")
intflow_velocities_at_boundary_faces = _make("intflow_velocities_at_boundary_faces", _p(
    "nx, ny, modvis, x, xp, xe, ye, xk, yk, u, v, ue, ve, un, vn, Uce, Vcn"), "mod_intflow.f90:692-787")
intflow_boundary_simplec = _make("intflow_boundary_simplec", _p("nx, ny, modvis, due, dve, dun, dvn, de, dn"),
                                 "mod_intflow.f90:791-877")
intflow_extrapolate_u_v_to_fictitious = _make("intflow_extrapolate_u_v_to_fictitious", _p(
    "nx, ny, modvis, x, xp, xk, yk, u, v"), "mod_intflow.f90:881-964")
intflow_time_cycle_update = _make("intflow_time_cycle_update", _p(
    "nx, ny, x, xp, u, gamma, Rg, P0, T0, uin, vin, pin, Tin, Mw, plin, pina, p"),
    "mod_intflow.f90:1106-1134 (thermomodel and iflow members as plain arguments)")
