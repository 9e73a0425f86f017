"""Writes oracle/orc_ns_mms.h: the Navier-Stokes manufactured solution and its
source term for the oracle's own workload callbacks (test infrastructure;
the product derives its copy separately, so the oracle does not take its
boundary data or source from the code under test).

The source is s = -div F(U, grad U) for the physical flux of the reference's
navier_stokes::Flux (navier_stokes.hpp:916-973) with unit reference
parameters (Re = Eu = e_coeff = 1) and constant viscosity: inviscid flux,
Stokes stress tau = mu (grad v + grad v^T) - 2/3 mu div v I, and the heat
flux as the reference forms it, q = mu gamma / Pr (grad E - v_k grad v_k)
(navier_stokes.hpp:700-746). The residual adds -s phi, so the manufactured
state solves the continuous steady problem.

Fields (x, y in [0, 1]^2):
    rho = 1 + A sin(2 pi x) sin(2 pi y)
    u   = u0 (1 + A cos(2 pi x) sin(2 pi y))
    v   = v0 (1 + A sin(2 pi x) cos(2 pi y))
    p   = pinf (1 + A cos(2 pi x) cos(2 pi y))

Run from this folder: python gen_ns_mms.py > orc_ns_mms.h
"""
import sympy as sp


def derive():
    x, y = sp.symbols("x y", real=True)
    gamma, Pr, mu, pinf, A, u0, v0 = sp.symbols("gamma Pr mu pinf A u0 v0", positive=True)
    k = 2 * sp.pi
    sx, cx, sy, cy = sp.sin(k * x), sp.cos(k * x), sp.sin(k * y), sp.cos(k * y)
    rho = 1 + A * sx * sy
    vel = (u0 * (1 + A * cx * sy), v0 * (1 + A * sx * cy))
    p = pinf * (1 + A * cx * cy)
    rhoE = p / (gamma - 1) + rho * (vel[0] ** 2 + vel[1] ** 2) / 2
    Etot = rhoE / rho
    X = (x, y)
    dv = [[sp.diff(vel[i], X[j]) for j in range(2)] for i in range(2)]
    divv = dv[0][0] + dv[1][1]
    tau = [[mu * (dv[i][j] + dv[j][i]) - (2 * mu * divv / 3 if i == j else 0) for j in range(2)]
           for i in range(2)]
    heat = [mu * gamma / Pr * (sp.diff(Etot, X[j]) - vel[0] * dv[0][j] - vel[1] * dv[1][j]) for j in range(2)]

    def flux(eq, j):
        if eq == 0:
            return rho * vel[j]
        if eq in (1, 2):
            i = eq - 1
            return rho * vel[i] * vel[j] + (p if i == j else 0) - tau[i][j]
        return vel[j] * (rhoE + p) - heat[j] - vel[0] * tau[0][j] - vel[1] * tau[1][j]

    state = [rho, rho * vel[0], rho * vel[1], rhoE]
    source = [-(sp.diff(flux(eq, 0), x) + sp.diff(flux(eq, 1), y)) for eq in range(4)]
    return state, source


def c_function(name, exprs):
    subs, outs = sp.cse(exprs)
    body = [f"static inline void {name}(double x, double y, const double* prm, double* out) {{",
            "  const double gamma = prm[0], Pr = prm[1], mu = prm[2], pinf = prm[3], A = prm[4], u0 = prm[5],"
            " v0 = prm[6];",
            "  (void)gamma; (void)Pr; (void)mu; (void)pinf; (void)A; (void)u0; (void)v0;"]
    body += [f"  const double {s} = {sp.ccode(e)};" for s, e in subs]
    body += [f"  out[{i}] = {sp.ccode(e)};" for i, e in enumerate(outs)]
    body.append("}")
    return "\n".join(body)


def main():
    state, source = derive()
    print("/* Written by oracle/gen_ns_mms.py (sympy); test infrastructure, do not edit. */")
    print("/* prm = {gamma, Pr, mu, pinf, A, u0, v0} */")
    print("#pragma once")
    print("#include <math.h>")
    print(c_function("orc_ns_mms_state_eval", state))
    print(c_function("orc_ns_mms_source_eval", source))


if __name__ == "__main__":
    main()
