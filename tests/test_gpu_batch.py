"""Batches of independent problems (one context, one launch per kernel for
all parts) against the same problems solved one context at a time: the
residual and Jacobian blocks of each part are its standalone ones, and Newton
and explicit solves of the batch land on the standalone solutions."""
import numpy as np
import pytest
import torch

import iceicle_b200 as ib
from specs import BURGERS, Spec

pytestmark = pytest.mark.gpu


def _parts(p=2, g=2):
    """uneven meshes and coefficients: linear advection-diffusion (b = 0) and Burgers"""
    return [
        Spec(pde=BURGERS, nx=3, ny=5, g=g, p=p, mu=0.05, a=(0.6, 0.8), b=(0.0, 0.0), perturb=0.05, seed=1),
        Spec(pde=BURGERS, nx=6, ny=4, g=g, p=p, mu=1e-3, a=(-1.0, 0.2), b=(0.0, 0.0), perturb=0.08, seed=2,
             dirichlet=[("constant", [1, -0.4])]),
        Spec(pde=BURGERS, nx=2, ny=2, g=g, p=p, mu=0.02, a=(0.0, 0.0), b=(1.0, 0.5), perturb=0.0, seed=3,
             bct=(3, 2, 4, 3)),
    ]


def _setup(specs):
    ctxs = [s.context() for s in specs]
    return ctxs, ib.batch(ctxs)


@pytest.mark.parametrize("pg", [(1, 1), (2, 2), (3, 2)], ids=["p1g1", "p2g2", "p3g2"])
def test_batch_residual_and_jacobian_are_the_parts(pg):
    specs = _parts(*pg)
    ctxs, b = _setup(specs)
    rng = np.random.default_rng(5)
    us = [s.state(rng) for s in specs]
    ub = torch.from_numpy(np.concatenate(us)).cuda()
    rb = torch.empty_like(ub)
    b.form_residual(ub, rb)
    off = 0
    for s, c, u in zip(specs, ctxs, us):
        du = torch.from_numpy(u).cuda()
        r = torch.empty_like(du)
        c.form_residual(du, r)
        assert torch.equal(rb[off:off + s.N], r), (s.nx, s.ny)
        off += s.N
    # Jacobian: the batch's block rows are the parts' block rows (shifted columns)
    Lb = b.layout
    bs2 = Lb.block_size ** 2
    vb = torch.empty(Lb.nnz_blocks * bs2, dtype=torch.float64, device="cuda")
    b.form_jacobian_fd(ub, rb, vb)
    rp_b, ci_b = b.jacobian_pattern()
    e0 = 0
    for s, c, u in zip(specs, ctxs, us):
        L = c.layout
        v = torch.empty(L.nnz_blocks * bs2, dtype=torch.float64, device="cuda")
        du = torch.from_numpy(u).cuda()
        c.form_jacobian_fd(du, torch.empty_like(du), v)
        rp, ci = c.jacobian_pattern()
        for e in range(L.n_elem):
            assert np.array_equal(ci_b[rp_b[e0 + e]:rp_b[e0 + e + 1]] - e0, ci[rp[e]:rp[e + 1]])
        kb0 = rp_b[e0]
        assert torch.equal(vb[kb0 * bs2:(kb0 + rp[-1]) * bs2], v)
        e0 += L.n_elem
    assert b.elem_offsets[-1] == Lb.n_elem


def test_batch_newton_matches_the_parts():
    """one Newton solve of the batch (one line search and one stopping test for
    the concatenated residual) lands on every part's standalone solution"""
    specs = _parts(2, 2)
    ctxs, b = _setup(specs)
    rng = np.random.default_rng(6)
    us = [0.2 * s.state(rng) for s in specs]
    opt = ib.default_newton_options()
    opt.tau_abs = 1e-12
    ub = torch.from_numpy(np.concatenate(us)).cuda()
    rep = b.newton_solve(ub, opt)
    assert rep.converged
    off = 0
    for s, c, u in zip(specs, ctxs, us):
        du = torch.from_numpy(u.copy()).cuda()
        assert c.newton_solve(du, opt).converged
        a, bb = du.cpu().numpy(), ub[off:off + s.N].cpu().numpy()
        assert np.linalg.norm(a - bb) <= 1e-10 * max(np.linalg.norm(a), np.linalg.norm(u))
        off += s.N


def test_batch_explicit_matches_the_parts():
    specs = _parts(2, 2)
    ctxs, b = _setup(specs)
    rng = np.random.default_rng(7)
    us = [s.state(rng) for s in specs]
    opt = ib.default_explicit_options(scheme=1, timestep=0, dt=1e-3, termination=0, ntime=3)
    ub = torch.from_numpy(np.concatenate(us)).cuda()
    b.explicit_solve(ub, opt)
    off = 0
    for s, c, u in zip(specs, ctxs, us):
        du = torch.from_numpy(u.copy()).cuda()
        c.explicit_solve(du, opt)
        a, bb = du.cpu().numpy(), ub[off:off + s.N].cpu().numpy()
        assert np.abs(a - bb).max() <= 1e-13 * np.abs(a).max()
        off += s.N


def test_batch_refuses_mixed_orders():
    a = Spec(pde=BURGERS, nx=2, ny=2, p=1).context()
    c = Spec(pde=BURGERS, nx=2, ny=2, p=2).context()
    with pytest.raises(ib.IcxError):
        ib.batch([a, c])
