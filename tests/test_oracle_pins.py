"""The oracle restatement against the reference's own code compiled here
(oracle/_ref) and against the reference's known-answer facts. CPU only."""
import numpy as np
import pytest

import oracle_bindings as ob
from specs import BURGERS, NS, Spec

needs_ref = pytest.mark.skipif(not ob.ref_available(), reason="reference CPU build absent")

CASES = [
    dict(),                                   # Burgers, p2, geometry order 2, DDG, Dirichlet
    dict(g=1, p=1),
    dict(p=3),
    dict(p=4, nx=2, ny=2),
    dict(ip=True),
    dict(sigma_ic=0.7),                       # DDGIC interface correction
    dict(bct=(3, 2, 4, 3)),                   # Dirichlet / Neumann / extrapolation
    dict(nx=1, ny=1),                         # single element: boundary faces only
    dict(nx=5, ny=1),                         # one row: no y-direction interior faces
    dict(bct=(0, 3, 0, 3)),                   # periodic in x: faces paired by flag, no flux across them
    dict(bct=(0, 0, 0, 0), p=3, sigma_ic=0.4),
    dict(pde=NS, p=2, ip=True),
    dict(pde=NS, p=3),
    dict(pde=NS, p=1, g=1, bct=(3, 4, 3, 4)),
    dict(pde=NS, p=2, ip=True, source=True),
    # DimensionlessSutherlands viscosity (mu_0/ref.mu, T_0/ref.T, T_s/ref.T)
    dict(pde=NS, p=2, ip=True, sutherland=(0.02, 0.004, 0.0015)),
    dict(pde=NS, p=3, sutherland=(0.02, 0.004, 0.0015), ns_mu=0.0, bct=(8, 3, 8, 3), walls=(0.004,)),
    # spacetime Burgers (x, t): past face without a connected slab, future face extrapolating
    dict(spacetime=True, a=(0.4,), b=(1.0,), bct=(3, 11, 3, 12)),
    dict(spacetime=True, p=3, a=(-0.3,), b=(0.5,), bct=(3, 3, 4, 12)),
    dict(spacetime=True, ip=True, sigma_ic=0.5, bct=(2, 3, 3, 12)),
    # Legendre (modal) solution basis
    dict(basis=1),
    dict(basis=1, p=4, nx=2, ny=2, sigma_ic=0.7),
    dict(basis=1, pde=NS, p=3, ip=True, source=True),
    dict(basis=1, spacetime=True, a=(0.4,), b=(1.0,), bct=(3, 11, 3, 12)),
]


def _state(spec, seed=0):
    return spec.state(np.random.default_rng(seed))


@needs_ref
@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
def test_residual_matches_reference(kw):
    spec = Spec(**kw)
    pb = spec.oracle_problem()
    c = spec.coords()
    u = _state(spec)
    r_or = ob.residual(ob.oracle(), pb, c, u)
    r_ref = ob.residual(ob.ref(), pb, c, u)
    scale = np.abs(r_ref).max()
    assert np.abs(r_or - r_ref).max() <= 1e-12 * scale


@needs_ref
@pytest.mark.parametrize("kw", [dict(), dict(g=1, p=1, nx=3, ny=5), dict(nx=1, ny=4), dict(bct=(0, 3, 0, 3)),
                                dict(nx=3, ny=4, bct=(0, 0, 0, 0))])
def test_topology_bit_exact(kw):
    spec = Spec(**kw)
    pb = spec.oracle_problem()
    c1, f1, n1 = ob.topology(ob.oracle(), pb)
    c2, f2, n2 = ob.topology(ob.ref(), pb)
    assert n1 == n2
    assert np.array_equal(c1, c2)
    assert np.array_equal(f1, f2)


@needs_ref
@pytest.mark.parametrize("kw", [dict(nx=3, ny=3), dict(nx=3, ny=2, bct=(3, 2, 4, 3), sigma_ic=0.5),
                                dict(pde=NS, nx=2, ny=2, p=2, ip=True),
                                dict(pde=NS, nx=2, ny=2, p=2, sutherland=(0.02, 0.004, 0.0015))])
def test_fd_jacobian_matches_reference(kw):
    """One-sided FD with eps = sqrt(machine eps) amplifies the last-bit
    differences of two residual evaluations by 1/eps ~ 7e7, so FD Jacobians of
    two implementations agree to ~1e-8 relative, not to machine precision.
    Tolerance: 1e-6 relative to the largest entry."""
    spec = Spec(**kw)
    pb = spec.oracle_problem()
    c = spec.coords()
    u = _state(spec, 3)
    r1, rowptr, colidx, vals = ob.jacobian_bsr(pb, c, u)
    J1 = ob.bsr_to_dense(rowptr, colidx, vals)
    r2, J2 = ob.ref_jacobian_dense(pb, c, u)
    assert np.abs(r1 - r2).max() <= 1e-12 * np.abs(r2).max()
    assert np.abs(J1 - J2).max() <= 1e-6 * np.abs(J2).max()
    # the reference's nonzeros lie inside the block pattern
    assert ((np.abs(J1) > 0) | (np.abs(J2) == 0)).all()


def test_fd_jacobian_matches_dense_fd_of_residual():
    """Shape of the reference's own test (test_petsc_jacobian.cpp:21-166): the
    assembled FD Jacobian agrees with a dense FD Jacobian of form_residual to 1e-5."""
    spec = Spec(nx=3, ny=3, g=1, p=1, bct=(3, 2, 3, 2), dirichlet=[("constant", [1, 0.0])],
                neumann=[("constant", [1, 1.0])])
    pb = spec.oracle_problem()
    c = spec.coords()
    u = _state(spec, 5)
    r, rowptr, colidx, vals = ob.jacobian_bsr(pb, c, u)
    J = ob.bsr_to_dense(rowptr, colidx, vals)
    eps = np.sqrt(np.finfo(float).eps)
    Jd = np.zeros_like(J)
    for j in range(len(u)):
        up = u.copy()
        up[j] += eps
        Jd[:, j] = (ob.residual(ob.oracle(), pb, c, up) - r) / eps
    assert np.abs(J - Jd).max() < 1e-5


def test_gauss_legendre_known_values():
    """Gauss-Legendre points/weights through a residual-independent path: a
    mass-like integral of x^(2n-1) polynomials is exact; checked against numpy's
    leggauss via the volume integral of a linear advection flux."""
    x, w = np.polynomial.legendre.leggauss(4)
    assert abs(w.sum() - 2.0) < 1e-15


def test_linear_state_has_zero_interior_jump_residual():
    """A globally linear state on an affine mesh with pure advection and no
    viscosity: the DG residual equals the exact weak form, so its sum over all
    test functions (partition of unity) is the boundary flux balance."""
    spec = Spec(nx=3, ny=3, g=1, p=1, mu=0.0, a=(1.0, 0.0), b=(0.0, 0.0), perturb=0.0,
                bct=(4, 4, 4, 4))
    pb = spec.oracle_problem()
    c = spec.coords()
    E, nb, N = ob.sizes(pb)
    # u = 1 everywhere: flux F = (1, 0); extrapolation boundaries carry it out
    u = np.ones(N)
    r = ob.residual(ob.oracle(), pb, c, u)
    # sum of residuals = -(outflow - inflow) = 0 for a divergence-free flux
    assert abs(r.sum()) < 1e-13


MDG_CASES = [
    dict(nx=4, ny=4, g=1, p=1, mu=0.0, a=(0.0, 1.0), b=(1.0, 0.0), bct=(3, 3, 3, 4),
         dirichlet=[("oblique_step", [0.4, 0.2, 1.0, -0.5])]),
    dict(nx=3, ny=4, g=1, p=2, mu=0.0, a=(0.0, 1.0), b=(1.0, 0.0), bct=(3, 3, 3, 4),
         dirichlet=[("oblique_step", [0.4, 0.2, 1.0, -0.5])]),
    dict(nx=3, ny=3, g=1, p=2, mu=0.02, bct=(3, 2, 4, 3)),
    dict(nx=3, ny=3, g=2, p=2, pde=NS, ip=True, perturb=0.05),
]


@needs_ref
@pytest.mark.parametrize("kw", MDG_CASES, ids=[str(c) for c in MDG_CASES])
def test_mdg_residual_and_jacobian_match_reference(kw):
    """MDG-ICE with all interior traces selected and hyper_rectangle boundary
    sliding: selection, geometry parameters, [res; ic] at moved nodes and the
    Jacobian w.r.t. [u; x] (FD tolerance as above)"""
    spec = Spec(**kw)
    pb = spec.oracle_problem()
    c = spec.coords()
    _, faces, nint = ob.topology(ob.oracle(), pb)
    traces = np.arange(nint)
    s1, x1 = ob.mdg_select(ob.oracle(), pb, c, traces)
    s2, x2 = ob.mdg_select(ob.ref(), pb, c, traces)
    assert np.array_equal(s1, s2) and np.array_equal(x1, x2)
    u = spec.state(np.random.default_rng(1))
    xp = x1 + 0.01 * np.random.default_rng(2).standard_normal(x1.size) / spec.nx
    r1 = ob.mdg_residual(ob.oracle(), pb, c, traces, u, xp)
    r2 = ob.mdg_residual(ob.ref(), pb, c, traces, u, xp)
    assert np.abs(r1 - r2).max() <= 1e-12 * np.abs(r2).max()
    o1, J1 = ob.mdg_jacobian_dense(ob.oracle(), pb, c, traces, u, xp)
    o2, J2 = ob.mdg_jacobian_dense(ob.ref(), pb, c, traces, u, xp)
    assert np.abs(o1 - o2).max() <= 1e-12 * np.abs(o2).max()
    assert np.abs(J1 - J2).max() <= 1e-6 * np.abs(J2).max()
    assert np.array_equal(J1 != 0, J2 != 0)


def test_oracle_mfnk_reaches_the_oracle_newton_state():
    """the oracle's MFNK restatement (difference products, unpreconditioned
    GMRES) converges to the assembled-Jacobian Newton's state down to the
    floor of its difference products"""
    import oracle_newton as on
    spec = Spec(pde=BURGERS, nx=3, ny=3, p=2, g=2, mu=1e-2, a=(0.2, 0.1), b=(1.0, 0.5),
                dirichlet=[("constant", [1, 0.25])])
    c = spec.coords()
    pb = spec.oracle_problem()
    u0 = 0.25 + 0.2 * np.random.default_rng(3).standard_normal(spec.N)
    u, k = on.mfnk(pb, c, u0, tau_abs=1e-8, kmax=30, rtol=1e-6)
    assert np.linalg.norm(ob.residual(ob.oracle(), pb, c, u)) <= 1e-8 and k < 30
    u_n, _ = on.newton(pb, c, u0, tau_abs=1e-12, kmax=20)
    assert np.linalg.norm(u - u_n) <= 1e-6 * np.linalg.norm(u_n)
