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


def mdg_layout(pb, coord, traces, hyper=True):
    """(selected nodes, parameter offsets cols[nsel + 1]) of an MDG selection"""
    import ctypes as C
    nn = (pb.nx * pb.geo_order + 1) * (pb.ny * pb.geo_order + 1)
    tr = np.ascontiguousarray(traces, dtype=np.int32)
    sel = np.zeros(nn, dtype=np.int32)
    cols = np.zeros(nn + 1, dtype=np.int32)
    f = ob.oracle().fn("mdg_layout")
    n = f(C.byref(pb), ob._ptr(coord), len(tr), ob._ptr(tr), int(hyper), ob._ptr(sel), ob._ptr(cols))
    assert n >= 0
    return sel[:n].copy(), cols[:n + 1].copy()


def mdg_jacobian_sparse(pb, coord, traces, u, x, hyper=True):
    """[res; ic] and the sparse Jacobian (CSR) w.r.t. [u; x] of the oracle
    (form_petsc_jacobian_fd + form_petsc_mdg_jacobian_fd)"""
    import ctypes as C
    E, nb, N = ob.sizes(pb)
    neq = ob.neq(pb)
    sel, cols = mdg_layout(pb, coord, traces, hyper)
    nres, ncol = N + len(sel) * neq, N + len(x)
    tr = np.ascontiguousarray(traces, dtype=np.int32)
    bs = nb * neq
    cap = 5 * E * bs * bs + 64 * len(sel) * (bs + 4) + 1024
    f = ob.oracle().fn("mdg_jacobian_coo")
    f.restype = C.c_longlong
    while True:
        rows = np.zeros(cap, dtype=np.int32)
        cls = np.zeros(cap, dtype=np.int32)
        vals = np.zeros(cap)
        out = np.zeros(nres)
        n = f(C.byref(pb), ob._ptr(coord), len(tr), ob._ptr(tr), int(hyper), ob._ptr(np.ascontiguousarray(u)),
              ob._ptr(np.ascontiguousarray(x)), ob._ptr(out), C.c_longlong(cap), ob._ptr(rows), ob._ptr(cls),
              ob._ptr(vals))
        assert n >= 0
        if n <= cap:
            break
        cap = int(n)
    J = sp.coo_matrix((vals[:n], (rows[:n], cls[:n])), shape=(nres, ncol)).tocsr()
    return out, J


def _coords_from_x(pb, coord0, sel, cols, x):
    """mesh nodes with the selected nodes' free coordinates from x (the
    fixed coordinates of a boundary node stay where they are)"""
    c = coord0.reshape(-1, 2).copy()
    for k, node in enumerate(sel):
        free = [d for d in range(2) if not _fixed(pb, node, d)]
        for i, d in enumerate(free):
            c[node, d] = x[cols[k] + i]
    return c.reshape(coord0.shape)


def _fixed(pb, node, d):
    """hyper_rectangle: the coordinate d of a node of the order-1 lattice index on the box is fixed"""
    if node >= (pb.nx + 1) * (pb.ny + 1):
        return False
    ix, iy = node % (pb.nx + 1), node // (pb.nx + 1)
    return (ix in (0, pb.nx)) if d == 0 else (iy in (0, pb.ny))


class ExplicitSubproblem:
    """the explicitly formed CorriganLM subproblem (corrigan_lm.hpp:426-530)
    of one configuration: (J^T J + diag(lambda_u |J_col|, lambda_b |J_col|)
    + lambda_lag |r| K^T K + lambda_el) p = J^T r, over the state unknowns and
    the free coordinates of the selected nodes. K^T K is formed as the
    reference forms it: its loop assigns KTK[i, j] = K[k, i] K[k, j] for every
    k in turn, so the last basis function's row k = ng - 1 is what remains
    (corrigan_lm.hpp:463-469)."""

    def __init__(self, pb, coord, traces):
        self.pb, self.traces = pb, traces
        self.E, self.nb, self.N = ob.sizes(pb)
        g = pb.geo_order
        self.ng = (g + 1) ** 2
        self.sel, self.cols = mdg_layout(pb, coord, traces)
        inv = {int(n): k for k, n in enumerate(self.sel)}
        free = [[d for d in range(2) if not _fixed(pb, int(n), d)] for n in self.sel]
        conn, _, _ = ob.topology(ob.oracle(), pb)
        self.coord0 = np.ascontiguousarray(coord)
        ng, N = self.ng, self.N

        def geo_pairs(e):
            """(row, col) positions of the free coordinates of every pair of selected nodes of element e"""
            out = []
            for il in range(ng):
                ki = inv.get(int(conn[e, il]))
                if ki is None:
                    continue
                for jl in range(ng):
                    kj = inv.get(int(conn[e, jl]))
                    if kj is None:
                        continue
                    for iv in range(len(free[ki])):
                        for jv in range(len(free[kj])):
                            out.append((il, jl, N + self.cols[ki] + iv, N + self.cols[kj] + jv))
            return out

        self.pairs = [geo_pairs(e) for e in range(self.E)]

    def state(self, xv):
        return np.ascontiguousarray(_coords_from_x(self.pb, self.coord0, self.sel, self.cols, xv))

    def linearise(self, u, x):
        """([res; ic], J) at (u, x)"""
        return mdg_jacobian_sparse(self.pb, self.state(x), self.traces, u, x)

    def cg_K(self, cw):
        import ctypes as C
        K = np.zeros((self.E, self.ng, self.ng))
        assert ob.oracle().fn("cg_stiffness")(C.byref(self.pb), ob._ptr(cw), ob._ptr(K)) == 0
        return K

    def min_det(self, cw):
        import ctypes as C
        m = np.zeros(self.E)
        assert ob.oracle().fn("min_detj")(C.byref(self.pb), ob._ptr(cw), ob._ptr(m)) == 0
        return m

    def system(self, out, J, x, lu, lb, lambda_lag, lam_el):
        """(M, rhs) of the subproblem at the linearisation (out, J) and nodes x"""
        N, ng = self.N, self.ng
        ncol = J.shape[1]
        rnorm = np.linalg.norm(out)
        Jt = J.T.tocsr()
        A = (Jt @ J).tocoo()
        cn = np.sqrt(np.asarray(J.multiply(J).sum(axis=0)).ravel())
        d = np.concatenate([lu * cn[:N], lb * cn[N:]])
        rr, cc, vv = [A.row], [A.col], [A.data]
        rr.append(np.arange(ncol)); cc.append(np.arange(ncol)); vv.append(d)
        Kall = self.cg_K(self.state(x))
        ri, ci, vi = [], [], []
        for e in range(self.E):
            Kl = Kall[e]
            KTK = np.outer(Kl[ng - 1], Kl[ng - 1])
            for il, jl, r, c in self.pairs[e]:
                ri.append(r); ci.append(c); vi.append(KTK[il, jl] * lambda_lag * rnorm)
            if lam_el[e] > 0.0:
                for il, jl, r, c in self.pairs[e]:
                    if il == jl:
                        ri.append(r); ci.append(c); vi.append(lam_el[e])
        rr.append(np.array(ri, dtype=np.int64)); cc.append(np.array(ci, dtype=np.int64)); vv.append(np.array(vi))
        M = sp.coo_matrix((np.concatenate(vv), (np.concatenate(rr), np.concatenate(cc))), shape=(ncol, ncol)).tocsc()
        return M, Jt @ out


def lm_explicit(pb, coord, traces, u0, x0, kmax=5, lambda_u=1e-7, lambda_b=1e-2, lambda_lag=1e-5, tau_abs=1e-10,
                max_rejections=20, history=None):
    """CorriganLM::solve with the explicitly formed subproblem
    (corrigan_lm.hpp:363-717, explicitly_form_subproblem = true, Corrigan line
    search): the ExplicitSubproblem system solved exactly (sparse LU),
    u <- u - alpha p_u, x <- x - alpha p_x, acceptance when no element inverts
    and |r_step| < 10 |r_old|, the lambda updates and the element-wise
    regularisation of the reference. Returns (u, x, residual norm history,
    alpha history)."""
    u, x = np.array(u0, dtype=float), np.array(x0, dtype=float)
    sub = ExplicitSubproblem(pb, coord, traces)
    E, N = sub.E, sub.N
    out, J = sub.linearise(u, x)
    hist = [np.linalg.norm(out)]
    alphas = []
    lu, lb, lu_min = lambda_u, lambda_b, lambda_u
    lam_el = np.zeros(E)
    k, rejects = 0, 0
    while k < kmax and hist[-1] > tau_abs:
        rnorm = np.linalg.norm(out)
        M, rhs = sub.system(out, J, x, lu, lb, lambda_lag, lam_el)
        p = spla.spsolve(M, rhs)
        state = sub.state
        min_det = sub.min_det
        last = {}

        def phi(a):
            o = ob.mdg_residual(ob.oracle(), pb, state(x - a * p[N:]), traces, u - a * p[:N], x - a * p[N:])
            v = np.linalg.norm(o[:N]) + np.linalg.norm(o[N:])
            last["v"], last["x"] = v, x - a * p[N:]
            return v
        alpha = corrigan_ls(phi)
        mins = min_det(state(last["x"]))
        reset = False
        for e in range(E):
            if mins[e] < 0.0:
                reset = True
                lam_el[e] = lb if lam_el[e] == 0 else lam_el[e] * max(1.5, abs(mins[e]))
        if not reset and last["v"] < 10 * rnorm:
            u, x = u - alpha * p[:N], x - alpha * p[N:]
            lu, lb = max(lu_min, 0.55 * lu), max(last["v"], 0.55 * lb)
            lam_el[lam_el > 0] /= 1.5
            rejects = 0
            alphas.append(alpha)
        else:
            lu, lb = lu * 1.8, lb * 1.8
            rejects += 1
            if rejects > max_rejections:
                break
            continue
        out, J = sub.linearise(u, x)
        hist.append(np.linalg.norm(out))
        if history is not None:
            history.append((hist[-1], alpha))
        k += 1
    return u, x, hist, alphas
