"""Explicit time stepping on the GPU (C ABI) against the oracle, which is
pinned to the reference's own ExplicitEuler / RK3TVD / RK3SSP: same mesh,
state, timestep rule and termination; FP64, 1e-12 relative to the largest
entry of the final state."""
import numpy as np
import pytest
import torch

import iceicle_b200 as ib
import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

RUNS = [
    (0, 0, 2e-3, 0.0, 0, 3, 0.0),
    (1, 0, 2e-3, 0.0, 0, 3, 0.0),
    (2, 0, 2e-3, 0.0, 0, 3, 0.0),
    (0, 1, 0.0, 0.3, 0, 4, 0.0),
    (1, 1, 0.0, 0.3, 1, 0, 0.01),
    (2, 1, 0.0, 0.5, 1, 0, 0.01),
]


def _opts(scheme, dk, dt, cfl, tk, nt, tf):
    return ib.default_explicit_options(scheme=scheme, timestep=dk, dt=dt, cfl=cfl, termination=tk, ntime=nt,
                                       tfinal=tf)


@pytest.mark.parametrize("run", RUNS, ids=[str(r) for r in RUNS])
@pytest.mark.parametrize("geo", [dict(g=2, p=2), dict(g=1, p=3, perturb=0.0)], ids=["g2p2", "g1p3"])
def test_explicit_burgers_matches_oracle(run, geo):
    spec = Spec(pde=BURGERS, nx=3, ny=3, mu=0.01, a=(0.3, -0.2), b=(1.0, 0.5), **geo)
    c = spec.coords()
    pb = spec.oracle_problem()
    u0 = spec.state(np.random.default_rng(3))
    uo, so, to = ob.explicit_solve(ob.oracle(), pb, c, u0, *run)
    ctx = spec.context(c)
    du = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.explicit_solve(du, _opts(*run))
    assert rep.steps == so and abs(rep.time - to) <= 1e-14 * max(to, 1.0)
    u = du.cpu().numpy()
    assert np.abs(u - uo).max() <= 1e-12 * np.abs(uo).max()


def test_explicit_ns_tvd_matches_oracle():
    spec = Spec(pde=NS, nx=3, ny=2, g=2, p=2, ip=True, source=True, perturb=0.05)
    c = spec.coords()
    pb = spec.oracle_problem()
    u0 = spec.state(np.random.default_rng(4))
    uo, _, _ = ob.explicit_solve(ob.oracle(), pb, c, u0, 1, 0, 1e-4, 0.0, 0, 2, 0.0)
    ctx = spec.context(c)
    du = torch.from_numpy(u0.copy()).cuda()
    ctx.explicit_solve(du, _opts(1, 0, 1e-4, 0.0, 0, 2, 0.0))
    u = du.cpu().numpy()
    assert np.abs(u - uo).max() <= 1e-12 * np.abs(uo).max()


def test_mass_inverse_apply_matches_oracle_mass_matrices():
    spec = Spec(pde=NS, nx=3, ny=3, g=2, p=3, ip=True, perturb=0.08)
    c = spec.coords()
    M = ob.mass_matrices(ob.oracle(), spec.oracle_problem(), c)
    r = np.random.default_rng(9).standard_normal(spec.N)
    ref = np.stack([np.linalg.solve(M[e], r.reshape(spec.E, spec.nb, 4)[e]) for e in range(spec.E)]).reshape(-1)
    ctx = spec.context(c)
    dr = torch.from_numpy(r).cuda()
    out = torch.empty_like(dr)
    ctx.mass_inverse_apply(dr, out)
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-11 * np.abs(ref).max()


def test_cfl_timestep_refused_without_wave_speed():
    spec = Spec(pde=NS, nx=2, ny=2, g=1, p=1, ip=True, perturb=0.0)
    ctx = spec.context()
    du = torch.from_numpy(spec.state(np.random.default_rng(1))).cuda()
    with pytest.raises(ib.IcxError):
        ctx.explicit_solve(du, _opts(1, 1, 0.0, 0.3, 0, 1, 0.0))
