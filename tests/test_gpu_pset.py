"""Sets of independent problems of uneven size and basis order
(icx_pset_*): each part solved by its own Newton iteration inside the set
equals the same part solved alone (icx_newton_solve).

* residual of the set = each part's own residual (1e-14 of its largest entry);
* Newton (Wolfe line search, GMRES(30) + block-ILU(0)) on a set of linear
  advection-diffusion parts of orders 1-4 and nonlinear viscous Burgers parts:
  every part converges, with the Newton iteration count of its own solve, its
  GMRES iteration total within 2 of it (per-part reductions are summed in
  another order than the single solve's), and its state within 1e-10 of its
  own solve's (relative to the larger L2 norm of that state and the initial
  state: the Burgers parts' steady state is u = 0);
* the same set in mixed precision reaches the FP64 states within 1e-10;
* the Arnoldi steps of the set are replayed from CUDA graphs;
* the same with one Gram-Schmidt pass per step (gmres_cgs_refine = 0).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _parts():
    import iceicle_b200.workloads as w
    specs = w.batched_problem_specs(10, seed=77, n_range=(3, 11))
    parts, u0 = [], []
    for sp in specs:
        c, u = w.advection_diffusion_problem(sp)
        parts.append(c)
        u0.append(u)
    for n, p in ((6, 2), (5, 3), (7, 1)):
        wl = w.burgers_config(nx=n, ny=n + 1, p=p, geo_order=1)
        parts.append(wl.ctx)
        u0.append(wl.u0)
    return parts, u0


@pytest.fixture(scope="module")
def problem_set():
    import iceicle_b200 as ib
    parts, u0 = _parts()
    ps = ib.ProblemSet(parts)
    assert len({c.layout.nbasis for c in parts}) >= 4  # every order 1-4 present
    return ps, parts, u0


def test_set_residual_is_each_parts_residual(problem_set):
    ps, parts, u0 = problem_set
    u = torch.from_numpy(ps.gather(u0)).cuda()
    r = torch.full_like(u, float("nan"))
    ps.residual(u, r)
    torch.cuda.synchronize()
    r = r.cpu().numpy()
    for k, c in enumerate(parts):
        uk = torch.from_numpy(u0[k]).cuda()
        rk = torch.empty_like(uk)
        c.form_residual(uk, rk)
        torch.cuda.synchronize()
        ref = rk.cpu().numpy()
        assert np.abs(ps.part(r, k) - ref).max() <= 1e-14 * max(np.abs(ref).max(), 1e-300), k


def _newton(ps, parts, u0, precision, refine=1):
    import iceicle_b200 as ib
    o = ib.default_newton_options()
    o.precision = precision
    o.gmres_cgs_refine = refine
    u = torch.from_numpy(ps.gather(u0)).cuda()
    reps, stats = ps.newton_solve(u, o)
    return u.cpu().numpy(), reps, stats, o


@pytest.mark.parametrize("refine", [1, 0], ids=["cgs2", "cgs1"])
def test_set_newton_equals_solving_each_part_alone(problem_set, refine):
    import iceicle_b200 as ib
    ps, parts, u0 = problem_set
    u, reps, stats, o = _newton(ps, parts, u0, 0, refine)
    assert stats.orders >= 4
    assert stats.graph_launches > 0
    for k, c in enumerate(parts):
        assert reps[k].converged, k
        uk = torch.from_numpy(u0[k].copy()).cuda()
        rk = c.newton_solve(uk, o)
        assert rk.converged
        assert reps[k].iterations == rk.iterations, (k, reps[k].iterations, rk.iterations)
        assert abs(reps[k].linear_iterations_total - rk.linear_iterations_total) <= 2, k
        ref = uk.cpu().numpy()
        scale = max(np.linalg.norm(ref), np.linalg.norm(u0[k]))
        assert np.linalg.norm(ps.part(u, k) - ref) <= 1e-10 * scale, k


def test_set_mixed_precision_reaches_fp64_states(problem_set):
    ps, parts, u0 = problem_set
    u64, _, _, _ = _newton(ps, parts, u0, 0)
    u32, reps, _, _ = _newton(ps, parts, u0, 1)
    for k in range(len(parts)):
        assert reps[k].converged
        a, b = ps.part(u64, k), ps.part(u32, k)
        assert np.linalg.norm(a - b) <= 1e-10 * max(np.linalg.norm(a), np.linalg.norm(u0[k])), k
