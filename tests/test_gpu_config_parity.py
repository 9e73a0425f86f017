"""Parity at the benchmark workloads' own sizes, CUDA path (through the C ABI)
against the C oracle on the same mesh nodes and states.

  * Navier-Stokes manufactured solution, 128 x 128 quads, p = 3, geometry
    order 2 (1,048,576 unknowns): the residual at 1e-12 of its largest entry;
    the Newton solve to |r| <= 1e-10 with every iterate's residual norm
    re-evaluated by the oracle, and the converged state a root of the
    oracle's residual.
  * the same physics on 32 x 32 quads: the first Newton step du of the GPU
    (FD Jacobian, GMRES to 1e-12) satisfies the oracle's Jacobian system to
    the finite-difference accuracy of two independent Jacobians.
  * viscous Burgers 32 x 32, p = 2: the whole Newton solve (Wolfe line
    search) against the oracle Newton (sparse direct solves): residual
    histories while |r| >> roundoff, converged state to 1e-10 of the initial
    state's L2 norm (the steady state of this problem is u = 0, so a norm
    relative to the converged state would compare roundoff with roundoff).

The inputs are built on each side independently: the oracle side takes mesh
nodes, basis-node coordinates and boundary/source callbacks from the oracle
library (tests/specs.py); the GPU side from the product's workload builders
(iceicle_b200.workloads), which are what bench.py times."""
import numpy as np
import pytest
import torch

import oracle_bindings as ob
import oracle_newton as on
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu


def _ns_spec(n):
    return Spec(pde=NS, nx=n, ny=n, p=3, g=2, ip=True, source=True, perturb=0.05, seed=4321)


def _ns_workload(n):
    from iceicle_b200.workloads import ns_mms_config
    return ns_mms_config(nx=n, ny=n, p=3, geo_order=2)


def _same_inputs(spec, wl):
    """the oracle-built nodes and state equal the product-built ones"""
    c = spec.coords()
    assert np.array_equal(c, wl.coords)
    u = spec.mms_state(c)
    assert np.abs(u - wl.u0).max() <= 1e-15 * np.abs(wl.u0).max()
    return c, u


def test_ns_128x128_p3_residual_full_size():
    spec, wl = _ns_spec(128), _ns_workload(128)
    c, u = _same_inputs(spec, wl)
    du = torch.from_numpy(wl.u0).cuda()
    dr = torch.full_like(du, float("nan"))
    wl.ctx.form_residual(du, dr)
    torch.cuda.synchronize()
    r = dr.cpu().numpy()
    ref = ob.residual(ob.oracle(), spec.oracle_problem(), c, wl.u0)
    assert np.isfinite(r).all()
    assert np.abs(r - ref).max() <= 1e-12 * np.abs(ref).max()


def test_ns_128x128_p3_roe_residual_full_size():
    """the same workload with the Roe flux the configuration names (parity
    unpinned against the reference, which has no Roe flux: here against the
    oracle's restatement of the published algorithm)"""
    import iceicle_b200 as ib
    from iceicle_b200.workloads import ns_mms_config
    spec = Spec(pde=NS, nx=128, ny=128, p=3, g=2, ip=True, source=True, perturb=0.05, seed=4321, ns_flux=2)
    wl = ns_mms_config(nx=128, ny=128, p=3, geo_order=2, conv_flux=ib.FLUX_ROE)
    c, u = _same_inputs(spec, wl)
    du = torch.from_numpy(wl.u0).cuda()
    dr = torch.full_like(du, float("nan"))
    wl.ctx.form_residual(du, dr)
    torch.cuda.synchronize()
    ref = ob.residual(ob.oracle(), spec.oracle_problem(), c, wl.u0)
    assert np.abs(dr.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_ns_256x256_p2_residual_full_size():
    """the learned-preconditioner workload's mesh and order (256 x 256, p = 2,
    2,359,296 unknowns) at Re = 300, at the workload's state with a seeded 1 %
    multiplicative perturbation: the manufactured state itself is nearly a
    root (its residual is ~1e-2 of the flux terms, so 1e-12 of it would be
    below the roundoff of the terms)"""
    from iceicle_b200.workloads import ns_mms_config
    spec = Spec(pde=NS, nx=256, ny=256, p=2, g=2, ip=True, source=True, perturb=0.05, seed=4321, ns_mu=1.0 / 300)
    wl = ns_mms_config(nx=256, ny=256, p=2, geo_order=2, mu=1.0 / 300)
    c = spec.coords()
    assert np.array_equal(c, wl.coords)
    u = wl.u0 * (1.0 + 0.01 * np.random.default_rng(17).standard_normal(wl.u0.size))
    du = torch.from_numpy(u).cuda()
    dr = torch.full_like(du, float("nan"))
    wl.ctx.form_residual(du, dr)
    torch.cuda.synchronize()
    ref = ob.residual(ob.oracle(), spec.oracle_problem(), c, u)
    assert np.abs(dr.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_ns_128x128_p3_newton_iterates_full_size():
    """one Newton step per call (Wolfe line search, GMRES(30) + block-ILU(0)
    to 1e-12): each iterate's residual norm as the GPU reports it equals the
    oracle's residual norm at that iterate, and the last iterate is a root of
    the oracle's residual to the Newton tolerance"""
    import iceicle_b200 as ib
    spec, wl = _ns_spec(128), _ns_workload(128)
    c, _ = _same_inputs(spec, wl)
    pb = spec.oracle_problem()
    du = torch.from_numpy(wl.u0.copy()).cuda()
    o = ib.default_newton_options()
    o.kmax, o.tau_abs, o.gmres_rtol, o.gmres_max_it = 1, 1e-10, 1e-12, 20000
    norms = []
    for k in range(8):
        u_k = du.cpu().numpy()
        r_or = ob.residual(ob.oracle(), pb, c, u_k)
        rep = wl.ctx.newton_solve(du, o)
        # the GPU's residual at the start of this call is the oracle's
        assert abs(rep.residual_history[0] - np.linalg.norm(r_or)) <= 1e-12 * max(np.linalg.norm(r_or), 1.0)
        norms.append(np.linalg.norm(r_or))
        if rep.residual_history[0] <= o.tau_abs:
            break
    assert norms[-1] <= 1e-10, norms
    assert len(norms) >= 3, norms  # it really iterated


def test_ns_32x32_p3_first_newton_step():
    """du from the GPU FD Jacobian and GMRES (rtol 1e-12) solves the oracle's
    FD Jacobian system: the two Jacobians agree to the ~1e-8 relative
    accuracy of one-sided differences, so the system residual is bounded by
    that, not by roundoff"""
    import scipy.sparse as sp
    spec, wl = _ns_spec(32), _ns_workload(32)
    c, _ = _same_inputs(spec, wl)
    L = wl.ctx.layout
    bs = L.block_size
    u = torch.from_numpy(wl.u0).cuda()
    res = torch.empty_like(u)
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    wl.ctx.form_jacobian_fd(u, res, vals)
    x = torch.zeros_like(u)
    wl.ctx.gmres_solve(vals, res, x, restart=30, maxit=20000, rtol=1e-12, preconditioner=2)
    torch.cuda.synchronize()
    du_g = x.cpu().numpy()
    r_or, rowptr, colidx, v_or = ob.jacobian_bsr(spec.oracle_problem(), c, wl.u0)
    assert np.abs(res.cpu().numpy() - r_or).max() <= 1e-12 * np.abs(r_or).max()
    A = sp.bsr_matrix((v_or, colidx, rowptr), shape=(L.n_dof, L.n_dof))
    rel = np.linalg.norm(A @ du_g - r_or) / np.linalg.norm(r_or)
    assert rel <= 1e-6, rel
    # and the blocks themselves at the FD tolerance used throughout
    vg = vals.cpu().numpy().reshape(v_or.shape)
    assert np.abs(vg - v_or).max() <= 1e-6 * np.abs(v_or).max()


def _burgers_inputs():
    """viscous Burgers 32 x 32 p = 2 workload, built on the oracle side:
    u0 = sin(2 pi x) sin(2 pi y) at the basis nodes + N(0, 1e-3), seed 1234"""
    spec = Spec(pde=BURGERS, nx=32, ny=32, p=2, g=2, mu=1e-2, a=(0.0, 0.0), b=(1.0, 0.5), perturb=0.0,
                dirichlet=[("constant", [1, 0.0])])
    c = spec.coords()
    pb = spec.oracle_problem()
    xy = ob.basis_node_coords(pb, c)
    rng = np.random.default_rng(1234)
    u0 = np.sin(2 * np.pi * xy[..., 0]) * np.sin(2 * np.pi * xy[..., 1])
    u0 = u0.reshape(-1) + rng.normal(0.0, 1e-3, size=u0.size)
    return spec, c, pb, u0


def test_burgers_32x32_p2_newton_matches_oracle_newton():
    import iceicle_b200 as ib
    from iceicle_b200.workloads import burgers_config
    spec, c, pb, u0 = _burgers_inputs()
    wl = burgers_config()
    assert np.array_equal(c, wl.coords)
    assert np.abs(u0 - wl.u0).max() <= 1e-15
    u_or, hist_or = on.newton(pb, c, u0, tau_abs=1e-10, kmax=20, linesearch="wolfe")
    o = ib.default_newton_options()
    o.tau_abs, o.kmax, o.gmres_rtol, o.gmres_max_it = 1e-10, 20, 1e-12, 20000
    du = torch.from_numpy(wl.u0.copy()).cuda()
    rep = wl.ctx.newton_solve(du, o)
    assert rep.converged
    hist = list(rep.residual_history[:rep.iterations + 1])
    assert hist_or[-1] <= 1e-10
    for a, b in zip(hist, hist_or):
        if b > 1e-6:
            assert abs(a - b) <= 1e-5 * b, (hist, hist_or)
    u = du.cpu().numpy()
    scale = max(np.linalg.norm(u_or), np.linalg.norm(u0))
    assert np.linalg.norm(u - u_or) <= 1e-10 * scale, np.linalg.norm(u - u_or) / scale
