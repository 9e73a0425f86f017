"""Oracle Newton (test infrastructure): PetscNewton::solve
(src/solvers/include/iceicle/petsc_newton.hpp:205-329) restated over the oracle
residual and FD Jacobian, with a sparse direct linear solve, and the
reference's Wolfe / Corrigan line searches
(src/solvers/include/iceicle/nonlinear_solver_utils.hpp:83-191)."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle_bindings as ob

SQEPS = np.sqrt(np.finfo(float).eps)


def _fd(f, eps, x):
    a = f(x)
    b = f(x + eps)
    return (b - a) / eps


def zoom(f, lo, hi, kmax, c1, c2):
    for _ in range(kmax):
        phi_lo, dphi_lo = f(lo), _fd(f, SQEPS, lo)
        phi_hi, dphi_hi = f(hi), _fd(f, SQEPS, hi)
        d1 = dphi_lo + dphi_hi - 3 * (phi_lo - phi_hi) / (lo - hi)
        d2 = np.sqrt(max(d1 * d1 - dphi_lo * dphi_hi, 1e-8))
        d2 = np.copysign(d2, hi - lo)
        aj = hi - (hi - lo) * ((dphi_hi + d2 - d1) / (dphi_hi - dphi_lo + 2 * d2))
        phi_aj = f(aj)
        dphi_0 = _fd(f, SQEPS, 0.0)
        if phi_aj > f(0.0) + c1 * aj * dphi_0 or phi_aj >= phi_lo:
            hi = aj
        else:
            dphi_aj = _fd(f, SQEPS, aj)
            if abs(dphi_aj) <= -c2 * dphi_0:
                return aj
            if dphi_aj * (hi - lo) >= 0:
                hi = lo
            lo = aj
    return 0.5 * (lo + hi)


def wolfe_ls(f, alpha_max=10.0, alpha1=1.0, kmax=20, c1=1e-4, c2=0.9):
    a_im1, a_i = 0.0, alpha1
    phi_0 = f(0.0)
    dphi_0 = _fd(f, SQEPS, 0.0)
    for k in range(kmax):
        phi_i, phi_im1 = f(a_i), f(a_im1)
        if phi_i > phi_0 + c1 * a_i * dphi_0 or (phi_i >= phi_im1 and k > 0):
            return zoom(f, a_im1, a_i, kmax, c1, c2)
        dphi_i = _fd(f, SQEPS, a_i)
        if abs(dphi_i) <= -c2 * dphi_0:
            return a_i
        if dphi_i >= 0:
            return zoom(f, a_i, a_im1, kmax, c1, c2)
        a_im1, a_i = a_i, 0.5 * (a_i + alpha_max)
    return a_i


def newton(pb, coord, u0, tau_abs=1e-10, kmax=20, linesearch=None):
    """returns (u, residual norm history)"""
    u = np.array(u0, dtype=np.float64)
    r, rowptr, colidx, vals = ob.jacobian_bsr(pb, coord, u)
    hist = [np.linalg.norm(r)]
    for _ in range(kmax):
        if hist[-1] <= tau_abs:
            break
        A = sp.bsr_matrix((vals, colidx, rowptr), shape=(u.size, u.size)).tocsc()
        du = spla.spsolve(A, r)
        alpha = 1.0
        if linesearch == "wolfe":
            def phi(a):
                v = np.linalg.norm(ob.residual(ob.oracle(), pb, coord, u - a * du))
                return v if np.isfinite(v) else 1e9
            alpha = wolfe_ls(phi)
        u = u - alpha * du
        r, rowptr, colidx, vals = ob.jacobian_bsr(pb, coord, u)
        hist.append(np.linalg.norm(r))
    return u, hist


def corrigan_ls(f, alpha_max=10.0, alpha1=1.0, kmax=20, alpha_min=0.0):
    a, b, alpha = alpha_min, alpha_max, alpha1
    for k in range(kmax):
        phi_0 = f(0.0)
        if k > 0:
            alpha = (a + b) / 2
        phi_star = f(alpha)
        if abs(phi_star) < abs(phi_0):
            if alpha == alpha1:
                break
            a = alpha
        else:
            b = alpha
    return alpha


def lm(pb, coord, traces, u0, x0, kmax=5, lambda_u=1e-7, lambda_b=1e-2, tau_abs=1e-10, linesearch=True):
    """CorriganLM::solve (corrigan_lm.hpp:363-717) with the matrix-free
    subproblem solved exactly; the regularisation follows the lambda updates.
    Returns (u, x, residual history)."""
    u, x = np.array(u0, dtype=float), np.array(x0, dtype=float)
    N = u.size
    out, J = ob.mdg_jacobian_dense(ob.oracle(), pb, coord, traces, u, x)
    hist = [np.linalg.norm(out)]
    lu, lb, lu_min = lambda_u, lambda_b, lambda_u
    k = 0
    rejects = 0
    while k < kmax and hist[-1] > tau_abs and rejects < 20:
        cn = np.linalg.norm(J, axis=0)
        d = np.concatenate([lu * cn[:N], np.maximum(lb, lb * cn[N:])])
        A = J.T @ J + np.diag(d)
        p = np.linalg.solve(A, J.T @ out)
        alpha, accept = 1.0, True
        if linesearch:
            last = {}

            def phi(a):
                o = ob.mdg_residual(ob.oracle(), pb, coord, traces, u - a * p[:N], x - a * p[N:])
                v = np.linalg.norm(o[:N]) + np.linalg.norm(o[N:])
                last["v"] = v
                last["x"] = x - a * p[N:]
                return v
            alpha = corrigan_ls(phi)
            accept = last["v"] < 10 * hist[-1]
            if accept:
                lu, lb = max(lu_min, 0.55 * lu), max(last["v"], 0.55 * lb)
            else:
                lu, lb = lu * 1.8, lb * 1.8
        if not accept:
            rejects += 1
            continue
        rejects = 0
        u, x = u - alpha * p[:N], x - alpha * p[N:]
        out, J = ob.mdg_jacobian_dense(ob.oracle(), pb, coord, traces, u, x)
        hist.append(np.linalg.norm(out))
        k += 1
    return u, x, hist


def mfnk(pb, coord, u0, tau_abs=1e-9, kmax=30, rtol=1e-6, restart=30, maxit=5000, linesearch=None, history=None):
    """MFNK::solve (src/solvers/include/iceicle/matrix_free_newton_krylov.hpp:
    219-365) without geometry unknowns, restated over the oracle residual: J p
    is the one-sided difference (R(u + eps p) - R(u)) / eps with the fixed
    eps = sqrt(machine epsilon) (jacobian_mf_op, :62-140), the Krylov solve is
    restarted GMRES without preconditioner from a zero guess, u <- u - alpha du,
    and the test |R| <= tau_abs runs after every step. Returns (u, steps)."""
    u = np.array(u0, dtype=float)
    r = ob.residual(ob.oracle(), pb, coord, u)
    k = 0
    for k in range(1, kmax + 1):
        r0 = r.copy()
        u_fix = u.copy()

        def mv(p):
            return (ob.residual(ob.oracle(), pb, coord, u_fix + SQEPS * p) - r0) / SQEPS

        A = spla.LinearOperator((len(u), len(u)), matvec=mv)
        du, _ = spla.gmres(A, r0, rtol=rtol, atol=0.0, restart=restart, maxiter=max(1, maxit // restart))
        alpha = 1.0
        if linesearch == "wolfe":
            def phi(a):
                v = np.linalg.norm(ob.residual(ob.oracle(), pb, coord, u - a * du))
                return v if np.isfinite(v) else 1e100
            alpha = wolfe_ls(phi)
        u = u - alpha * du
        r = ob.residual(ob.oracle(), pb, coord, u)
        if history is not None:
            history.append(float(np.linalg.norm(r)))
        if np.linalg.norm(r) <= tau_abs:
            break
    return u, k
