"""GPU FD Jacobian (BSR) and BSR SpMV through the C ABI against the oracle's
FD Jacobian with the reference perturbation scheme.

Tolerance: 1e-6 relative to the largest entry. One-sided differences with
eps = sqrt(machine eps) amplify last-bit differences between two residual
evaluations by ~1/eps, so two correct FD Jacobians agree to ~1e-8, not to
machine precision (the oracle and the reference's own build agree to 2e-8)."""
import numpy as np
import pytest
import torch

import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

CASES = [
    dict(nx=3, ny=3),
    dict(nx=4, ny=3, g=1, p=1),
    dict(nx=3, ny=2, p=3),
    dict(nx=3, ny=3, ip=True),
    dict(nx=3, ny=2, sigma_ic=0.5, bct=(3, 2, 4, 3)),
    dict(nx=1, ny=1),
    dict(nx=4, ny=1, p=1),
    dict(pde=NS, nx=2, ny=2, p=2, ip=True),
    dict(pde=NS, nx=2, ny=3, p=3, ip=True, source=True),
    dict(pde=NS, nx=2, ny=2, p=1, g=1, bct=(3, 4, 3, 4)),
    dict(pde=NS, nx=2, ny=2, p=2),
    dict(nx=3, ny=3, spacetime=True, a=(0.4,), b=(1.0,), bct=(3, 11, 3, 12)),
    dict(nx=3, ny=2, p=3, spacetime=True, a=(-0.3,), b=(0.5,), bct=(3, 3, 4, 12)),
    dict(nx=3, ny=3, basis=1),
    dict(pde=NS, nx=2, ny=2, p=2, ip=True, basis=1),
]


def gpu_jacobian(ctx, u):
    L = ctx.layout
    bs = L.block_size
    du = torch.from_numpy(u).cuda()
    dr = torch.full_like(du, float("nan"))
    dv = torch.full((L.nnz_blocks * bs * bs,), float("nan"), dtype=torch.float64, device="cuda")
    ctx.form_jacobian_fd(du, dr, dv)
    torch.cuda.synchronize()
    return dr.cpu().numpy(), dv.cpu().numpy().reshape(-1, bs, bs)


@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
def test_jacobian_parity(kw):
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(5))
    r_or, rowptr, colidx, v_or = ob.jacobian_bsr(spec.oracle_problem(), c, u)
    ctx = spec.context(c)
    rp, ci = ctx.jacobian_pattern()
    assert np.array_equal(rp, rowptr) and np.array_equal(ci, colidx)
    r, v = gpu_jacobian(ctx, u)
    assert np.isfinite(v).all(), "every block of the pattern must be written"
    assert np.abs(r - r_or).max() <= 1e-12 * np.abs(r_or).max()
    assert np.abs(v - v_or).max() <= 1e-6 * np.abs(v_or).max()


def test_spmv_matches_dense_product():
    spec = Spec(pde=NS, nx=3, ny=3, p=2, ip=True)
    ctx = spec.context()
    u = spec.state(np.random.default_rng(1))
    r, v = gpu_jacobian(ctx, u)
    rp, ci = ctx.jacobian_pattern()
    Jd = ob.bsr_to_dense(rp, ci, v)
    x = np.random.default_rng(2).standard_normal(Jd.shape[0])
    dv = torch.from_numpy(v.reshape(-1)).cuda()
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    ctx.bsr_spmv(dv, dx, dy)
    torch.cuda.synchronize()
    y = dy.cpu().numpy()
    ref = Jd @ x
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


def test_jacobian_times_direction_matches_residual_difference():
    """size-independent property on a larger mesh: J d ~ (R(u + h d) - R(u)) / h"""
    spec = Spec(pde=NS, nx=16, ny=16, p=3, ip=True, source=True)
    ctx = spec.context()
    rng = np.random.default_rng(9)
    u = spec.state(rng)
    r, v = gpu_jacobian(ctx, u)
    d = rng.standard_normal(u.size) * np.abs(u).mean()
    h = 1e-7
    du = torch.from_numpy(u + h * d).cuda()
    dr = torch.empty_like(du)
    ctx.form_residual(du, dr)
    dv = torch.from_numpy(v.reshape(-1)).cuda()
    jd = torch.empty_like(du)
    ctx.bsr_spmv(dv, torch.from_numpy(d).cuda(), jd)
    torch.cuda.synchronize()
    fd = (dr.cpu().numpy() - r) / h
    jdv = jd.cpu().numpy()
    assert np.linalg.norm(jdv - fd) <= 1e-4 * np.linalg.norm(fd)
