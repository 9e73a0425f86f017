"""GPU residual (through the C ABI) against the oracle on the same mesh,
coordinates and state: FP64, tolerance 1e-12 relative to the largest entry."""
import numpy as np
import pytest
import torch

import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

CASES = [
    dict(),
    dict(g=1, p=1),
    dict(p=3),
    dict(p=4, nx=3, ny=2),
    dict(ip=True),
    dict(sigma_ic=0.7),
    dict(bct=(3, 2, 4, 3)),
    dict(nx=1, ny=1),
    dict(nx=5, ny=1),
    dict(nx=1, ny=4, p=1),
    dict(pde=NS, p=2, ip=True),
    dict(pde=NS, p=3),
    dict(pde=NS, p=3, ip=True, source=True),
    dict(pde=NS, p=1, g=1, bct=(3, 4, 3, 4)),
    dict(pde=NS, p=4, g=2, nx=2, ny=3, ip=True),
    dict(nx=12, ny=9, p=2, perturb=0.2),
    dict(spacetime=True, a=(0.4,), b=(1.0,), bct=(3, 11, 3, 12)),
    dict(spacetime=True, p=3, a=(-0.3,), b=(0.5,), bct=(3, 3, 4, 12)),
    dict(spacetime=True, p=4, nx=3, ny=4, ip=True, sigma_ic=0.5, bct=(2, 3, 3, 12)),
    dict(basis=1),
    dict(basis=1, p=4, nx=3, ny=2, sigma_ic=0.7),
    dict(basis=1, pde=NS, p=3, ip=True, source=True),
    dict(basis=1, g=1, p=1, bct=(3, 2, 4, 3)),
    dict(pde=NS, p=2, ip=True, sutherland=(0.02, 0.004, 0.0015)),  # Sutherland viscosity
    dict(pde=NS, p=3, sutherland=(0.02, 0.004, 0.0015), ns_mu=0.0, bct=(8, 3, 8, 3), walls=(0.004,)),
    dict(bct=(0, 3, 0, 3)),                       # periodic pairs: no flux across them
    dict(bct=(0, 0, 0, 0), p=3, sigma_ic=0.4),
]


def _gpu_residual(ctx, u):
    du = torch.from_numpy(u).cuda()
    dr = torch.full_like(du, float("nan"))
    ctx.form_residual(du, dr)
    torch.cuda.synchronize()
    return dr.cpu().numpy()


@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
def test_residual_parity(kw):
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(11))
    r_or = ob.residual(ob.oracle(), spec.oracle_problem(), c, u)
    ctx = spec.context(c)
    r = _gpu_residual(ctx, u)
    assert np.isfinite(r).all()
    assert np.abs(r - r_or).max() <= 1e-12 * np.abs(r_or).max()


@pytest.mark.parametrize("bct", [(3, 3, 3, 3), (0, 3, 0, 3), (0, 0, 0, 0)])
def test_topology_and_pattern_bit_exact(bct):
    spec = Spec(nx=5, ny=4, bct=bct)
    ctx = spec.context()
    pb = spec.oracle_problem()
    c1, f1, n1 = ob.topology(ob.oracle(), pb)
    c2, f2, n2 = ctx.topology()
    assert n1 == n2 and np.array_equal(c1, c2) and np.array_equal(f1, f2)
    rp1, ci1 = ob.bsr_pattern(pb)
    rp2, ci2 = ctx.jacobian_pattern()
    assert np.array_equal(rp1, rp2) and np.array_equal(ci1, ci2)


def test_residual_repeatable_and_node_update():
    """same inputs give bit-identical outputs; moving nodes re-tabulates geometry"""
    spec = Spec(nx=6, ny=5, p=2)
    c = spec.coords()
    u = spec.state(np.random.default_rng(2))
    ctx = spec.context(c)
    r1 = _gpu_residual(ctx, u)
    r2 = _gpu_residual(ctx, u)
    assert np.array_equal(r1, r2)
    from iceicle_b200.workloads import perturb_smooth
    c2 = perturb_smooth(c, (spec.nx, spec.ny), 0.15, 99)
    ctx.set_coords(c2)
    r3 = _gpu_residual(ctx, u)
    r_or = ob.residual(ob.oracle(), spec.oracle_problem(), c2, u)
    assert np.abs(r3 - r_or).max() <= 1e-12 * np.abs(r_or).max()


def test_full_size_ns_properties():
    """NS manufactured-solution workload at benchmark size (128x128, p=3),
    properties beside the oracle comparison at this size
    (test_gpu_config_parity.py): deterministic, and the residual of the exact
    nodal state is small relative to that of a perturbed state (consistency
    of the manufactured source)."""
    from iceicle_b200.workloads import ns_mms_config
    wl = ns_mms_config(state_noise=0.0)
    r_exact = _gpu_residual(wl.ctx, wl.u0)
    wl2 = ns_mms_config(state_noise=1e-2)
    r_pert = _gpu_residual(wl2.ctx, wl2.u0)
    assert np.isfinite(r_exact).all() and np.isfinite(r_pert).all()
    assert np.linalg.norm(r_exact) < 0.05 * np.linalg.norm(r_pert)
    r_again = _gpu_residual(wl.ctx, wl.u0)
    assert np.array_equal(r_exact, r_again)
