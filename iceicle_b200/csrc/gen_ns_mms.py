"""Generates icx_ns_mms.h: a manufactured solution for the 2D compressible
Navier-Stokes workload and its source term s = -div F(U, grad U), derived
symbolically from the physical flux the kernels implement (inviscid flux plus
viscous stress and heat flux q = mu gamma / Pr (grad E - u_k grad u_k), unit
reference parameters so that Re = Eu = e_coeff = 1; navier_stokes.hpp:700-746,
916-973). The residual adds -s phi, so the exact state is a steady solution
of the continuous problem.

    rho = 1 + A sin(2 pi x) sin(2 pi y)
    u   = u0 (1 + A cos(2 pi x) sin(2 pi y))
    v   = v0 (1 + A sin(2 pi x) cos(2 pi y))
    p   = p_inf (1 + A cos(2 pi x) cos(2 pi y)),  p_inf = rho_inf |u_inf|^2 / (gamma M^2)

Run: python gen_ns_mms.py > icx_ns_mms.h
"""
import sympy as sp

x, y = sp.symbols("x y", real=True)
gamma, Pr, mu, pinf, A, u0, v0 = sp.symbols("gamma Pr mu pinf A u0 v0", real=True, positive=True)
pi2 = 2 * sp.pi
rho = 1 + A * sp.sin(pi2 * x) * sp.sin(pi2 * y)
u = u0 * (1 + A * sp.cos(pi2 * x) * sp.sin(pi2 * y))
v = v0 * (1 + A * sp.sin(pi2 * x) * sp.cos(pi2 * y))
p = pinf * (1 + A * sp.cos(pi2 * x) * sp.cos(pi2 * y))
rhoE = p / (gamma - 1) + rho * (u * u + v * v) / 2
U = [rho, rho * u, rho * v, rhoE]
vel = [u, v]
X = [x, y]
E = rhoE / rho
gv = [[sp.diff(vel[i], X[j]) for j in range(2)] for i in range(2)]
div = gv[0][0] + gv[1][1]
tau = [[mu * (gv[i][j] + gv[j][i]) - (sp.Rational(2, 3) * mu * div if i == j else 0) for j in range(2)] for i in range(2)]
q = [mu * gamma / Pr * (sp.diff(E, X[j]) - sum(vel[k] * gv[k][j] for k in range(2))) for j in range(2)]
F = [[None, None] for _ in range(4)]
for j in range(2):
    F[0][j] = rho * vel[j]
    for i in range(2):
        F[1 + i][j] = rho * vel[i] * vel[j] + (p if i == j else 0) - tau[i][j]
    F[3][j] = vel[j] * (rhoE + p) - (q[j] + sum(vel[i] * tau[i][j] for i in range(2)))
S = [-(sp.diff(F[k][0], x) + sp.diff(F[k][1], y)) for k in range(4)]

def emit(name, exprs):
    reps, red = sp.cse(exprs, optimizations="basic")
    lines = [f"static inline void {name}(double x, double y, double gamma, double Pr, double mu, double pinf,",
             "                                 double A, double u0, double v0, double* out) {",
             "  (void)gamma; (void)Pr; (void)mu;"]
    for s, e in reps:
        lines.append(f"  const double {s} = {sp.ccode(e)};")
    for k, e in enumerate(red):
        lines.append(f"  out[{k}] = {sp.ccode(e)};")
    lines.append("}")
    return "\n".join(lines)

print("// Generated by gen_ns_mms.py (sympy); do not edit by hand.")
print("// Manufactured Navier-Stokes solution (conservative variables) and its source.")
print("#pragma once")
print("#include <math.h>")
print(emit("icx_ns_mms_state", U))
print(emit("icx_ns_mms_source", S))
