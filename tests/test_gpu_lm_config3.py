"""MDG-ICE at the benchmark size: 64 x 64 quads, p = 1 and p = 2, oblique
shock of inviscid Burgers with interior nodes jittered by +-0.2 h, every
interior trace selected; CorriganLM with the explicitly formed subproblem
(J^T J + column-norm diagonal + lambda_lag |r| K^T K + element-wise
regularisation, ILU(0)-preconditioned GMRES to 1e-12) through icx_lm_solve,
against the oracle's restatement of CorriganLM::solve (corrigan_lm.hpp:363-717)
with the same subproblem solved by sparse LU.

Both sides run two LM iterations from the same state and nodes. Their FD
Jacobians are two independent one-sided-difference evaluations (they agree to
~1e-8 relative, the tolerance argued in test_gpu_jacobian.py), so the steps,
residual histories and node positions agree to 1e-6 relative; the GPU's
iterate is then pinned exactly: the oracle's [res; ic] at the GPU's state and
nodes equals the GPU's to 1e-12 of its largest entry."""
import numpy as np
import pytest
import torch

import oracle_bindings as ob
import oracle_newton as on
from specs import Spec

pytestmark = pytest.mark.gpu


def _jitter(coord, n, frac, seed):
    rng = np.random.default_rng(seed)
    out = coord.copy()
    for k in range(out.shape[0]):
        ix, iy = k % (n + 1), k // (n + 1)
        d = rng.uniform(-frac, frac, 2)
        if 0 < ix < n and 0 < iy < n:
            out[k] += d / n
    return np.ascontiguousarray(out)


@pytest.mark.parametrize("n,p", [(10, 1), (8, 2)])
def test_small_lm_explicit_matches_oracle(n, p):
    """the same configuration on small meshes, where the subproblem is well
    enough conditioned for GMRES to reach 1e-12: three LM iterations against
    the oracle at 1e-6 (two independent FD Jacobians)"""
    import iceicle_b200 as ib
    from iceicle_b200.workloads import mdg_ice_config
    wl, traces, x0 = mdg_ice_config(n=n, p=p)
    spec = Spec(nx=n, ny=n, g=1, p=p, mu=0.0, a=(0.0, 1.0), b=(1.0, 0.0), bct=(3, 3, 3, 4),
                dirichlet=[("oblique_step", [0.4, 0.2, 1.0, -0.5])], perturb=0.0)
    pb = spec.oracle_problem()
    c = _jitter(spec.coords(), n, 0.2, 99)
    assert np.array_equal(c, wl.coords)
    u_or, x_or, hist_or, _ = on.lm_explicit(pb, c, traces, wl.u0, x0, kmax=3)
    o = ib.default_lm_options()
    o.kmax, o.explicit_subproblem, o.gmres_rtol, o.gmres_max_it, o.gmres_restart = 3, 1, 1e-12, 20000, 60
    du = torch.from_numpy(wl.u0.copy()).cuda()
    x = x0.copy()
    rep = ib.lm_solve(wl.ctx, du, x, o)
    hist = list(rep.residual_history[:rep.iterations + 1])
    assert rep.linear_relres_max <= 1e-12, rep.linear_relres_max
    assert rep.iterations == len(hist_or) - 1, (hist, hist_or)
    for a, b in zip(hist, hist_or):
        assert abs(a - b) <= 1e-6 * b, (hist, hist_or)
    assert np.linalg.norm(x - x_or) <= 1e-6 * np.linalg.norm(x_or)


@pytest.mark.parametrize("p", [1, 2])
def test_config3_lm_explicit_matches_oracle(p):
    import iceicle_b200 as ib
    from iceicle_b200.workloads import mdg_ice_config
    n = 64
    wl, traces, x0 = mdg_ice_config(n=n, p=p)
    spec = Spec(nx=n, ny=n, g=1, p=p, mu=0.0, a=(0.0, 1.0), b=(1.0, 0.0), bct=(3, 3, 3, 4),
                dirichlet=[("oblique_step", [0.4, 0.2, 1.0, -0.5])], perturb=0.0)
    pb = spec.oracle_problem()
    c = _jitter(spec.coords(), n, 0.2, 99)
    assert np.array_equal(c, wl.coords)
    sel, x_or0 = ob.mdg_select(ob.oracle(), pb, c, traces)
    assert np.array_equal(x_or0, x0)
    xy = ob.basis_node_coords(pb, c).reshape(-1, 2)
    u0 = np.where(xy[:, 0] < 0.4 + 0.2 * xy[:, 1], 1.0, -0.5)
    assert np.array_equal(u0, wl.u0)
    kmax = 2
    u_or, x_or, hist_or, al_or = on.lm_explicit(pb, c, traces, u0, x0, kmax=kmax)
    o = ib.default_lm_options()
    o.kmax, o.explicit_subproblem, o.gmres_rtol, o.gmres_max_it, o.gmres_restart = kmax, 1, 1e-12, 20000, 60
    du = torch.from_numpy(u0.copy()).cuda()
    x = x0.copy()
    rep = ib.lm_solve(wl.ctx, du, x, o)
    hist = list(rep.residual_history[:rep.iterations + 1])
    assert rep.iterations == len(hist_or) - 1, (hist, hist_or)
    for a, b in zip(hist, hist_or):
        assert abs(a - b) <= 1e-6 * b, (hist, hist_or)
    assert np.linalg.norm(x - x_or) <= 1e-6 * np.linalg.norm(x_or)
    u = du.cpu().numpy()
    assert np.linalg.norm(u - u_or) <= 1e-6 * np.linalg.norm(u_or)
    # the GPU iterate is pinned: [res; ic] of the oracle at the GPU's (u, x)
    res = torch.empty_like(du)
    L = wl.ctx.layout
    nsel = len(sel)
    ic = torch.empty(nsel, dtype=torch.float64, device="cuda")
    wl.ctx.form_residual_mdg(du, x, res, ic)
    torch.cuda.synchronize()
    got = np.concatenate([res.cpu().numpy(), ic.cpu().numpy()])
    ref = ob.mdg_residual(ob.oracle(), pb, c, traces, u, x)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
