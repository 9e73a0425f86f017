"""GMRES / block preconditioners and the Newton solver on the GPU (C ABI),
against dense solves and the oracle Newton (PetscNewton::solve restated)."""
import numpy as np
import pytest
import torch

import iceicle_b200 as ib
import oracle_bindings as ob
import oracle_newton as on
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu


def _jac(ctx, u):
    L = ctx.layout
    bs = L.block_size
    du = torch.from_numpy(u).cuda()
    dr = torch.empty_like(du)
    dv = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    ctx.form_jacobian_fd(du, dr, dv)
    return dr, dv


@pytest.mark.parametrize("pc", [0, 1, 2], ids=["none", "block_jacobi", "block_ilu0"])
def test_gmres_matches_dense_solve(pc):
    spec = Spec(pde=NS, nx=4, ny=3, p=2, ip=True)
    ctx = spec.context()
    u = spec.state(np.random.default_rng(3))
    dr, dv = _jac(ctx, u)
    x = torch.zeros_like(dr)
    it, rr, ok = ctx.gmres_solve(dv, dr, x, restart=30, maxit=3000, rtol=1e-11, preconditioner=pc)
    assert ok, (it, rr)
    rp, ci = ctx.jacobian_pattern()
    bs = ctx.layout.block_size
    Jd = ob.bsr_to_dense(rp, ci, dv.cpu().numpy().reshape(-1, bs, bs))
    xr = np.linalg.solve(Jd, dr.cpu().numpy())
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr)


@pytest.mark.parametrize("shape", [(6, 1), (1, 5)])
def test_block_ilu0_is_exact_on_block_tridiagonal(shape):
    """one row (or column) of elements gives a block-tridiagonal Jacobian, on
    which block ILU(0) is the exact block LU: GMRES converges in one step"""
    spec = Spec(pde=NS, nx=shape[0], ny=shape[1], p=2, ip=True)
    ctx = spec.context()
    u = spec.state(np.random.default_rng(4))
    dr, dv = _jac(ctx, u)
    x = torch.zeros_like(dr)
    it, rr, ok = ctx.gmres_solve(dv, dr, x, restart=30, maxit=50, rtol=1e-10, preconditioner=2)
    assert ok and it == 1, (it, rr)


def test_preconditioners_reduce_iterations():
    spec = Spec(pde=BURGERS, nx=12, ny=12, p=2, mu=0.05)
    ctx = spec.context()
    u = spec.state(np.random.default_rng(6))
    dr, dv = _jac(ctx, u)
    its = []
    for pc in (0, 1, 2):
        x = torch.zeros_like(dr)
        it, rr, ok = ctx.gmres_solve(dv, dr, x, restart=30, maxit=5000, rtol=1e-8, preconditioner=pc)
        assert ok
        its.append(it)
    assert its[2] < its[1] <= its[0], its


def _newton_opts(**kw):
    o = ib.default_newton_options()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def test_newton_spacetime_burgers_slab_matches_oracle_newton():
    """one spacetime slab of viscous Burgers in (x, t): initial data and
    inflow as Dirichlet data, SPACETIME_FUTURE on top. Newton without line
    search on both sides; converged states agree to 1e-10 (L2, relative)"""
    spec = Spec(pde=BURGERS, nx=6, ny=4, p=2, g=2, mu=2e-2, a=(0.3,), b=(1.0,), spacetime=True,
                bct=(3, 3, 4, 12), dirichlet=[("constant", [1, 0.4])])
    c = spec.coords()
    ctx = spec.context(c)
    xy = ctx.basis_node_coords().reshape(-1, 2)
    u0 = 0.4 + 0.1 * np.sin(2 * np.pi * xy[:, 0]) + 1e-3 * np.random.default_rng(3).standard_normal(len(xy))
    u_or, hist_or = on.newton(spec.oracle_problem(), c, u0, tau_abs=1e-12, kmax=15)
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-12, kmax=15, linesearch=0, gmres_rtol=1e-13,
                                            gmres_max_it=5000))
    assert rep.converged, list(rep.residual_history[:rep.iterations + 1])
    u = du.cpu().numpy()
    assert np.linalg.norm(u - u_or) <= 1e-10 * np.linalg.norm(u_or)


def test_newton_burgers_matches_oracle_newton():
    """no line search, tight linear solves: both sides take the same Newton
    steps, so the residual histories agree while |r| >> roundoff and the
    converged states agree to 1e-10 (L2, relative)"""
    spec = Spec(pde=BURGERS, nx=6, ny=6, p=2, g=2, mu=1e-2, a=(0.0, 0.0), b=(1.0, 0.5),
                dirichlet=[("constant", [1, 0.0])])
    c = spec.coords()
    rng = np.random.default_rng(8)
    xy = None
    ctx = spec.context(c)
    xy = ctx.basis_node_coords().reshape(-1, 2)
    u0 = 0.5 * np.sin(2 * np.pi * xy[:, 0]) * np.sin(2 * np.pi * xy[:, 1]) + 1e-3 * rng.standard_normal(len(xy))
    u_or, hist_or = on.newton(spec.oracle_problem(), c, u0, tau_abs=1e-12, kmax=15)
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-12, kmax=15, linesearch=0, gmres_rtol=1e-13,
                                            gmres_max_it=5000))
    assert rep.converged, list(rep.residual_history[:rep.iterations + 1])
    hist = list(rep.residual_history[:rep.iterations + 1])
    for a, b in zip(hist, hist_or):
        if b > 1e-6:
            assert abs(a - b) <= 1e-6 * b, (hist, hist_or)
    u = du.cpu().numpy()
    assert np.linalg.norm(u - u_or) <= 1e-10 * max(np.linalg.norm(u_or), 1e-300) or \
        np.linalg.norm(u - u_or) <= 1e-12


def test_newton_with_gmres_restarts_matches_oracle():
    """short restarts force several GMRES cycles per Newton step: the Newton
    right-hand side must survive them (regression: it once shared a buffer
    with GMRES's restart residual)"""
    # non-zero boundary data so that the converged state is not ~0
    spec = Spec(pde=BURGERS, nx=6, ny=5, p=2, g=2, mu=1e-2, a=(0.2, 0.1), b=(1.0, 0.5),
                dirichlet=[("constant", [1, 0.25])])
    c = spec.coords()
    ctx = spec.context(c)
    u0 = 0.25 + 0.2 * np.random.default_rng(12).standard_normal(spec.N)
    u_or, hist_or = on.newton(spec.oracle_problem(), c, u0, tau_abs=1e-12, kmax=20)
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-12, kmax=20, linesearch=0, gmres_restart=3,
                                            gmres_rtol=1e-12, gmres_max_it=20000, preconditioner=1))
    assert rep.converged
    hist = list(rep.residual_history[:rep.iterations + 1])
    for a, b in zip(hist[:4], hist_or[:4]):
        assert abs(a - b) <= 1e-6 * b, (hist, hist_or)
    assert np.linalg.norm(du.cpu().numpy() - u_or) <= 1e-10 * np.linalg.norm(u_or)


def test_newton_ns_mms_with_linesearch_converges_to_oracle_state():
    spec = Spec(pde=NS, nx=4, ny=4, p=2, g=2, ip=True, source=True, perturb=0.05)
    c = spec.coords()
    ctx = spec.context(c)
    from iceicle_b200 import workload_fn
    import ctypes as C
    from iceicle_b200.workloads import ns_mms_params
    prm = ns_mms_params()
    f = workload_fn("ns_mms_state")
    xy = ctx.basis_node_coords().reshape(-1, 2)
    out = (C.c_double * 4)()
    pt = (C.c_double * 2)()
    u0 = np.zeros((len(xy), 4))
    for k in range(len(xy)):
        pt[0], pt[1] = xy[k]
        f(pt, out, C.cast(prm, C.c_void_p))
        u0[k] = out[:]
    u0 = (u0 * (1 + 1e-2 * np.random.default_rng(2).standard_normal(u0.shape))).reshape(-1)
    u_or, hist_or = on.newton(spec.oracle_problem(), c, u0, tau_abs=1e-11, kmax=20, linesearch="wolfe")
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=20, linesearch=1, gmres_rtol=1e-12,
                                            gmres_max_it=5000))
    assert rep.converged and rep.r_final <= 1e-11
    u = du.cpu().numpy()
    assert np.linalg.norm(u - u_or) <= 1e-10 * np.linalg.norm(u_or)


@pytest.mark.parametrize("pc", [1, 2])
def test_newton_mixed_precision_converges_to_fp64_oracle_state(pc):
    """precision = 1: SpMV and preconditioner read FP32 copies (FP32
    accumulation) inside FP64 Newton. The Newton residual is FP64, so the
    converged state is the FP64 one: within 1e-10 (L2, relative) of the
    oracle's, the same bar as the all-FP64 solve; only the inner iteration
    counts may differ."""
    spec = Spec(pde=NS, nx=4, ny=4, p=2, g=2, ip=True, source=True, perturb=0.05)
    c = spec.coords()
    ctx = spec.context(c)
    from iceicle_b200 import workload_fn
    import ctypes as C
    from iceicle_b200.workloads import ns_mms_params
    prm = ns_mms_params()
    f = workload_fn("ns_mms_state")
    xy = ctx.basis_node_coords().reshape(-1, 2)
    out = (C.c_double * 4)()
    pt = (C.c_double * 2)()
    u0 = np.zeros((len(xy), 4))
    for k in range(len(xy)):
        pt[0], pt[1] = xy[k]
        f(pt, out, C.cast(prm, C.c_void_p))
        u0[k] = out[:]
    u0 = (u0 * (1 + 1e-2 * np.random.default_rng(2).standard_normal(u0.shape))).reshape(-1)
    u_or, _ = on.newton(spec.oracle_problem(), c, u0, tau_abs=1e-11, kmax=20, linesearch="wolfe")
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=30, linesearch=1, gmres_rtol=1e-5,
                                            gmres_max_it=5000, preconditioner=pc, precision=1))
    assert rep.converged and rep.r_final <= 1e-11
    u = du.cpu().numpy()
    assert np.linalg.norm(u - u_or) <= 1e-10 * np.linalg.norm(u_or)


def test_newton_mixed_precision_burgers_ilu():
    """mixed precision on the 32 x 32 viscous Burgers configuration: converges
    in FP64 and lands on the all-FP64 solution. With zero Dirichlet data and
    no source the steady state is u = 0, so the difference is measured
    against the initial state's norm (1e-10); both solves run to
    |r| <= 1e-12 so that their states are comparable"""
    from iceicle_b200.workloads import burgers_config
    wl = burgers_config()
    u64 = torch.from_numpy(wl.u0.copy()).cuda()
    r64 = wl.ctx.newton_solve(u64, _newton_opts(tau_abs=1e-12))
    u32 = torch.from_numpy(wl.u0.copy()).cuda()
    r32 = wl.ctx.newton_solve(u32, _newton_opts(tau_abs=1e-12, precision=1))
    assert r64.converged and r32.converged and r32.r_final <= 1e-12
    a, b = u64.cpu().numpy(), u32.cpu().numpy()
    assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(wl.u0)


def test_mfnk_matches_the_oracle_mfnk():
    """matrix-free Newton-Krylov (no stored Jacobian, GMRES without
    preconditioner) against the oracle's restatement of the reference MFNK on
    a Burgers problem with nonzero boundary data. The Jacobian products are
    one-sided differences with the fixed eps = sqrt(machine epsilon), whose
    rounding floor (here |R| about 3e-9) bounds how far either solver can
    drive the residual, so both stop at |R| <= 1e-8. The residual histories
    agree while |R| is far above that floor (the two GMRES differ in their
    last digits), and the state lands on the oracle Newton's converged state
    to 1e-6 (L2, relative)."""
    spec = Spec(pde=BURGERS, nx=5, ny=4, p=2, g=2, mu=1e-2, a=(0.2, 0.1), b=(1.0, 0.5),
                dirichlet=[("constant", [1, 0.25])])
    c = spec.coords()
    pb = spec.oracle_problem()
    ctx = spec.context(c)
    u0 = 0.25 + 0.2 * np.random.default_rng(21).standard_normal(spec.N)
    hist_or = []
    on.mfnk(pb, c, u0, tau_abs=1e-8, kmax=30, rtol=1e-6, history=hist_or)
    u_newton, _ = on.newton(pb, c, u0, tau_abs=1e-12, kmax=20)
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.mfnk_solve(du, _newton_opts(tau_abs=1e-8, kmax=30, linesearch=0, gmres_rtol=1e-6,
                                          gmres_max_it=5000))
    assert rep.converged and rep.r_final <= 1e-8
    hist = list(rep.residual_history[1:rep.iterations + 1])
    assert len(hist) == len(hist_or), (hist, hist_or)
    for a_, b_ in zip(hist, hist_or):
        if b_ > 1e-5:
            assert abs(a_ - b_) <= 1e-3 * b_, (hist, hist_or)
    assert np.linalg.norm(du.cpu().numpy() - u_newton) <= 1e-6 * np.linalg.norm(u_newton)


def _ns_mms_state(ctx, noise, seed):
    from iceicle_b200 import workload_fn
    import ctypes as C
    from iceicle_b200.workloads import ns_mms_params
    prm = ns_mms_params()
    f = workload_fn("ns_mms_state")
    xy = ctx.basis_node_coords().reshape(-1, 2)
    out = (C.c_double * 4)()
    pt = (C.c_double * 2)()
    u0 = np.zeros((len(xy), 4))
    for k in range(len(xy)):
        pt[0], pt[1] = xy[k]
        f(pt, out, C.cast(prm, C.c_void_p))
        u0[k] = out[:]
    return (u0 * (1 + noise * np.random.default_rng(seed).standard_normal(u0.shape))).reshape(-1)


def test_mfnk_ns_with_linesearch_matches_assembled_newton():
    """MFNK with the Wolfe line search and the assembled-Jacobian Newton land
    on the same Navier-Stokes state. With total energy near 25 the floor of
    the difference products is |R| about 1e-6 here (the oracle MFNK stalls
    between 1e-6 and 3e-7), so MFNK stops at |R| <= 5e-6, where the oracle's
    state is 3e-8 from the converged one; the states agree to 1e-6 (L2,
    relative)."""
    spec = Spec(pde=NS, nx=3, ny=3, p=2, g=2, ip=True, source=True, perturb=0.05)
    ctx = spec.context()
    u0 = _ns_mms_state(ctx, 1e-2, 22)
    u1 = torch.from_numpy(u0.copy()).cuda()
    r1 = ctx.newton_solve(u1, _newton_opts(tau_abs=1e-8, kmax=30, gmres_rtol=1e-6, gmres_max_it=5000))
    u2 = torch.from_numpy(u0.copy()).cuda()
    r2 = ctx.mfnk_solve(u2, _newton_opts(tau_abs=5e-6, kmax=40, gmres_rtol=1e-6, gmres_max_it=5000))
    assert r1.converged and r2.converged
    a, b = u1.cpu().numpy(), u2.cpu().numpy()
    assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(a)


@pytest.mark.parametrize("pc,precision", [(2, 0), (2, 1), (1, 0), (4, 1), (0, 0)],
                         ids=["ilu0_fp64", "ilu0_mixed", "jacobi_fp64", "sweeps_mixed", "none_fp64"])
def test_newton_cuda_graphs_bit_identical(pc, precision):
    """the Arnoldi steps replayed as CUDA graphs launch the same kernels in the
    same order as the eager steps: the Newton iterates, GMRES counts and
    converged state are identical bit for bit, and graphs were replayed"""
    spec = Spec(pde=BURGERS, nx=8, ny=7, p=2, g=2, mu=1e-2, a=(0.0, 0.0), b=(1.0, 0.5),
                dirichlet=[("constant", [1, 0.0])])
    c = spec.coords()
    out = {}
    for graphs in (0, 1):
        ctx = spec.context(c)
        xy = ctx.basis_node_coords().reshape(-1, 2)
        u0 = 0.5 * np.sin(2 * np.pi * xy[:, 0]) * np.sin(2 * np.pi * xy[:, 1]) + \
            1e-3 * np.random.default_rng(8).standard_normal(len(xy))
        du = torch.from_numpy(u0).cuda()
        rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=15, preconditioner=pc, precision=precision,
                                                gmres_restart=10, gmres_rtol=1e-6, gmres_max_it=4000,
                                                cuda_graphs=graphs))
        assert rep.converged, list(rep.residual_history[:rep.iterations + 1])
        out[graphs] = (du.cpu().numpy(), rep.iterations, list(rep.linear_iterations[:rep.iterations]),
                       list(rep.residual_history[:rep.iterations + 1]), rep.graph_steps)
    (u0_, it0, lin0, h0, g0), (u1_, it1, lin1, h1, g1) = out[0], out[1]
    assert g0 == 0 and g1 > 0
    assert it0 == it1 and lin0 == lin1 and h0 == h1
    assert np.array_equal(u0_.view(np.uint64), u1_.view(np.uint64))


@pytest.mark.parametrize("precision,tile", [(0, 0), (1, 0), (1, 4)], ids=["fp64", "mixed", "mixed_tiled"])
def test_newton_matrix_free_operator_reaches_the_assembled_state(precision, tile):
    """matrix_free = 1: the GMRES operator is the residual's directional
    difference (h = sqrt(eps) (sqrt(n) + |u|) / |v|), the assembled FD
    Jacobian preconditions only. On the Navier-Stokes manufactured solution
    (line search, |R| <= 1e-11) it converges to the assembled Newton's state
    within 1e-10 (L2, relative), with GMRES iteration totals within 50 % of
    it (40 against 55 and 112 against 156 measured: the difference product
    is the residual's own derivative, not the element-wise FD Jacobian the
    preconditioner factors), and its Arnoldi steps (residual launches
    included) replay as graphs."""
    spec = Spec(pde=NS, nx=6, ny=5, p=2, g=2, ip=True, source=True, perturb=0.05)
    ctx = spec.context()
    u0 = _ns_mms_state(ctx, 1e-2, 23)
    out = {}
    for mf in (0, 1):
        du = torch.from_numpy(u0.copy()).cuda()
        rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=20, linesearch=1, gmres_rtol=1e-6,
                                                gmres_max_it=5000, precision=precision, ilu_tile=tile,
                                                matrix_free=mf))
        assert rep.converged and rep.r_final <= 1e-11, (mf, list(rep.residual_history[:rep.iterations + 1]))
        out[mf] = (du.cpu().numpy(), rep.linear_iterations_total, rep.graph_steps)
    (ua, ita, _), (um, itm, gm) = out[0], out[1]
    assert np.linalg.norm(um - ua) <= 1e-10 * np.linalg.norm(ua)
    assert abs(itm - ita) <= 0.5 * ita + 2, (itm, ita)
    assert gm > 0


def test_newton_bf16_factors_reach_the_fp64_state():
    """precision 3: tiled block-ILU(0) factors in BF16 (FP32 arithmetic), the
    rest as precision 1; with the matrix-free operator and without, Newton
    converges to the FP64 solve's state within 1e-10 (L2, relative)"""
    spec = Spec(pde=NS, nx=6, ny=5, p=2, g=2, ip=True, source=True, perturb=0.05)
    ctx = spec.context()
    u0 = _ns_mms_state(ctx, 1e-2, 23)
    du = torch.from_numpy(u0.copy()).cuda()
    r0 = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=20, linesearch=1, gmres_rtol=1e-6, gmres_max_it=5000))
    assert r0.converged
    ua = du.cpu().numpy()
    for mf in (0, 1):
        du = torch.from_numpy(u0.copy()).cuda()
        rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=20, linesearch=1, gmres_rtol=1e-6,
                                                gmres_max_it=5000, precision=3, ilu_tile=3, matrix_free=mf))
        assert rep.converged and rep.r_final <= 1e-11, (mf, list(rep.residual_history[:rep.iterations + 1]))
        assert np.linalg.norm(du.cpu().numpy() - ua) <= 1e-10 * np.linalg.norm(ua)
        assert rep.graph_steps > 0


@pytest.mark.parametrize("precision,tile,mf", [(0, 0, 0), (1, 0, 0), (3, 3, 1)], ids=["fp64", "mixed", "bf16_mf"])
def test_newton_single_gram_schmidt_pass_reaches_the_same_state(precision, tile, mf):
    """gmres_cgs_refine = 0: one classical Gram-Schmidt pass per Arnoldi step
    (PETSc's default GMRES orthogonalisation). Newton converges to the state
    of the two-pass FP64 solve within 1e-10 (L2, relative), and its graph
    replay is bit-identical to eager steps."""
    spec = Spec(pde=NS, nx=6, ny=5, p=2, g=2, ip=True, source=True, perturb=0.05)
    ctx = spec.context()
    u0 = _ns_mms_state(ctx, 1e-2, 23)
    du = torch.from_numpy(u0.copy()).cuda()
    r0 = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=20, linesearch=1, gmres_rtol=1e-6, gmres_max_it=5000))
    assert r0.converged
    ua = du.cpu().numpy()
    out = {}
    for graphs in (0, 1):
        du = torch.from_numpy(u0.copy()).cuda()
        rep = ctx.newton_solve(du, _newton_opts(tau_abs=1e-11, kmax=20, linesearch=1, gmres_rtol=1e-6,
                                                gmres_max_it=5000, precision=precision, ilu_tile=tile,
                                                matrix_free=mf, gmres_cgs_refine=0, cuda_graphs=graphs))
        assert rep.converged and rep.r_final <= 1e-11
        u = du.cpu().numpy()
        assert np.linalg.norm(u - ua) <= 1e-10 * np.linalg.norm(ua)
        out[graphs] = (u, list(rep.linear_iterations[:rep.iterations]), rep.graph_steps)
    assert out[1][2] > 0 and out[0][2] == 0
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0].view(np.uint64), out[1][0].view(np.uint64))
