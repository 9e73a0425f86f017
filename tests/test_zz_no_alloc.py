"""Allocation-free residual entry point (icx_form_residual_noalloc).

It serves callers that cannot allocate device memory while they evaluate
residuals (a host framework that owns the device memory pool and forbids other
allocations during a solve; a time-critical loop that must avoid cudaMalloc's
device-wide synchronisation). Its face scratch is a fixed 2^20-double device
array. Checked here through the C ABI against icx_form_residual on two calls in
a row and directly against the oracle's residual (tolerance 1e-12 relative to
the largest entry, as the other residual parity tests), and the size limit is
checked to fail cleanly.

This file is collected last so that a run that stops at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

import iceicle_b200 as ib
import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu


def _both(ctx, u):
    du = torch.from_numpy(u).cuda()
    r_ref = torch.full_like(du, float("nan"))
    r_new = torch.full_like(du, float("nan"))
    ctx.form_residual(du, r_ref)
    ctx.form_residual_noalloc(du, r_new)
    torch.cuda.synchronize()
    return r_ref.cpu().numpy(), r_new.cpu().numpy()


@pytest.mark.parametrize("kw", [dict(pde=NS, nx=32, ny=32, p=3, ip=True, source=True),
                                dict(pde=BURGERS, nx=16, ny=12, p=2, sigma_ic=0.7, bct=(3, 2, 4, 3))],
                         ids=["ns_p3_32x32", "burgers_ddgic"])
def test_noalloc_matches_residual_two_calls(kw):
    spec = Spec(**kw)
    ctx = spec.context()
    rng = np.random.default_rng(21)
    for _ in range(2):
        u = spec.state(rng)
        r_ref, r_new = _both(ctx, u)
        assert np.isfinite(r_new).all()
        assert np.abs(r_new - r_ref).max() <= 1e-12 * np.abs(r_ref).max()
    ctx.close()


@pytest.mark.parametrize("kw", [dict(pde=NS, nx=12, ny=10, p=3, ip=True, source=True),
                                dict(pde=BURGERS, nx=9, ny=7, p=4, sigma_ic=0.5, bct=(3, 2, 4, 3))],
                         ids=["ns_p3_12x10", "burgers_p4_ddgic"])
def test_noalloc_matches_oracle(kw):
    spec = Spec(**kw)
    c = spec.coords()
    ctx = spec.context(c)
    u = spec.state(np.random.default_rng(23))
    du = torch.from_numpy(u).cuda()
    dr = torch.full_like(du, float("nan"))
    ctx.form_residual_noalloc(du, dr)
    torch.cuda.synchronize()
    r = dr.cpu().numpy()
    r_or = ob.residual(ob.oracle(), spec.oracle_problem(), c, u)
    assert np.isfinite(r).all()
    assert np.abs(r - r_or).max() <= 1e-12 * np.abs(r_or).max()
    ctx.close()


def test_noalloc_rejects_oversized_problem():
    # 200x200 quads, p = 4, geometry order 2: 80,400 faces x 6 points x 4 equations > 2^20
    spec = Spec(pde=NS, nx=200, ny=200, p=4, g=2, ip=True, perturb=0.0)
    ctx = spec.context()
    n = ctx.layout.n_dof
    du = torch.zeros(n, dtype=torch.float64, device="cuda")
    dr = torch.zeros_like(du)
    with pytest.raises(ib.IcxError) as ei:
        ctx.form_residual_noalloc(du, dr)
    assert ei.value.status == 7  # ICX_ERR_SIZE
    assert "scratch" in str(ei.value)
    ctx.close()
