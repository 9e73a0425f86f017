"""The partitioned residual on the GPU: every rank's sub-mesh context
(iceicle_b200.partition) evaluated on one device, its ghost rows filled from
the neighbouring strips' owned rows by the plan's halo ranges (plain copies
stand in for the exchange between processes), must give owned entries
bit-identical to the global context's residual; the strip workload builder
must agree with the whole-mesh one."""
import numpy as np
import pytest
import torch

from iceicle_b200.partition import StripPlan, sub_coords
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

CASES = [
    dict(pde=BURGERS, nx=6, ny=9, p=2),
    dict(pde=NS, nx=5, ny=8, p=3, ip=True, source=True),
    dict(pde=NS, nx=4, ny=7, p=2),
]


@pytest.mark.parametrize("nranks", [2, 3, 4])
@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
def test_strip_residuals_match_global(kw, nranks):
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(4))
    bs = spec.nb * spec.neq
    glob = spec.context(c)
    du = torch.from_numpy(u).cuda()
    rg = torch.empty_like(du)
    glob.form_residual(du, rg)
    plans = [StripPlan(spec.nx, spec.ny, nranks, r, spec.g) for r in range(nranks)]
    # owned rows from the global state, ghost rows NaN until the exchange
    locs = []
    for p in plans:
        d0, d1 = p.global_dofs(bs)
        ul = torch.full((d1 - d0,), float("nan"), dtype=torch.float64, device="cuda")
        o0, o1 = p.owned_dofs(bs)
        ul[o0:o1] = du[d0 + o0:d0 + o1]
        locs.append(ul)
    for p, ul in zip(plans, locs):
        for peer, _, (r0, r1) in p.halo(bs):
            back = [h for h in plans[peer].halo(bs) if h[0] == p.rank][0]
            s0, s1 = back[1]
            ul[r0:r1] = locs[peer][s0:s1]
    torch.cuda.synchronize()
    for p, ul in zip(plans, locs):
        assert not torch.isnan(ul).any()
        sub = Spec(**dict(kw, ny=p.rows)).context(sub_coords(p, c))
        rl = torch.empty_like(ul)
        sub.form_residual(ul, rl)
        torch.cuda.synchronize()
        o0, o1 = p.owned_dofs(bs)
        ref = rg[p.j0 * spec.nx * bs:p.j1 * spec.nx * bs]
        assert torch.equal(rl[o0:o1].view(torch.int64), ref.view(torch.int64)), p.rank


def test_strip_workload_single_rank_is_whole_mesh():
    """the one-rank strip workload is the benchmark workload (same mesh,
    coordinates and residual at the same state)"""
    from iceicle_b200.workloads import ns_mms_config, ns_mms_strip_config
    a = ns_mms_config(nx=16, ny=16, p=3, geo_order=2)
    b = ns_mms_strip_config(StripPlan(16, 16, 1, 0, 2), p=3, geo_order=2)
    assert np.array_equal(a.coords, b.coords)
    u = torch.from_numpy(a.u0).cuda()
    ra, rb = torch.empty_like(u), torch.empty_like(u)
    a.ctx.form_residual(u, ra)
    b.ctx.form_residual(u, rb)
    torch.cuda.synchronize()
    assert torch.equal(ra.view(torch.int64), rb.view(torch.int64))
