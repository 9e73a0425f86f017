"""Navier-Stokes PDE-level boundaries (slip wall, no-slip isothermal wall,
WALL_GENERAL, Riemann far field; navier_stokes.hpp:976-1189) and the Roe
convective flux on the GPU, through the C ABI, against the oracle:
residuals at 1e-12 of the largest entry, FD Jacobians at 1e-6 (the one-sided
difference tolerance of test_gpu_jacobian.py). The oracle's boundary states
are pinned to the reference build (test_oracle_ns_bc_roe.py); the Roe flux
has no reference counterpart (parity unpinned: consistency and conservation
are checked there). Also: a Newton solve with the Roe flux on the
manufactured solution converges, and a uniform state on an unperturbed mesh
with extrapolation boundaries has a zero residual (free-stream preservation
of a consistent flux)."""
import numpy as np
import pytest
import torch

import oracle_bindings as ob
from specs import NS, Spec
from test_gpu_jacobian import gpu_jacobian
from test_gpu_residual import _gpu_residual
from test_oracle_ns_bc_roe import BC_CASES, FREE, WALL_T

pytestmark = pytest.mark.gpu

ROE_CASES = [
    dict(pde=NS, p=2, ip=True, ns_flux=2),
    dict(pde=NS, p=3, ns_flux=2, source=True),
    dict(pde=NS, p=1, g=1, ns_flux=2, bct=(3, 4, 3, 4)),
    dict(pde=NS, p=2, ns_flux=2, bct=(5, 7, 5, 6), bcf=(0, 0, 0, 1), walls=WALL_T, free_stream=FREE),
]


@pytest.mark.parametrize("kw", BC_CASES + ROE_CASES, ids=[f"bc{i}" for i in range(len(BC_CASES))] +
                         [f"roe{i}" for i in range(len(ROE_CASES))])
def test_residual_parity(kw):
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(4))
    r_or = ob.residual(ob.oracle(), spec.oracle_problem(), c, u)
    ctx = spec.context(c)
    r = _gpu_residual(ctx, u)
    assert np.isfinite(r).all()
    assert np.abs(r - r_or).max() <= 1e-12 * np.abs(r_or).max()


@pytest.mark.parametrize("kw", [dict(BC_CASES[0], nx=2, ny=2), dict(ROE_CASES[3], nx=2, ny=3)], ids=["bc", "roe"])
def test_jacobian_parity(kw):
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(5))
    r_or, rp, ci, v_or = ob.jacobian_bsr(spec.oracle_problem(), c, u)
    ctx = spec.context(c)
    r, v = gpu_jacobian(ctx, u)
    assert np.abs(r - r_or).max() <= 1e-12 * np.abs(r_or).max()
    assert np.abs(v - v_or).max() <= 1e-6 * np.abs(v_or).max()


@pytest.mark.parametrize("flux", [1, 2], ids=["van_leer", "roe"])
def test_uniform_state_has_zero_residual(flux):
    spec = Spec(pde=NS, nx=5, ny=4, p=2, g=1, perturb=0.0, ns_flux=flux, bct=(4, 4, 4, 4))
    ctx = spec.context()
    u = np.tile([1.0, 0.4, -0.3, 2.6], spec.N // 4)
    r = _gpu_residual(ctx, u)
    assert np.abs(r).max() <= 1e-13


def test_newton_with_roe_flux_converges():
    import iceicle_b200 as ib
    from iceicle_b200.workloads import ns_mms_config
    wl = ns_mms_config(nx=16, ny=16, p=2, conv_flux=ib.FLUX_ROE)
    o = ib.default_newton_options()
    o.tau_abs, o.gmres_rtol = 1e-10, 1e-8
    u = torch.from_numpy(wl.u0.copy()).cuda()
    rep = wl.ctx.newton_solve(u, o)
    assert rep.converged, list(rep.residual_history[:rep.iterations + 1])
    # the converged state is a root of the oracle's Roe residual
    spec = Spec(pde=NS, nx=16, ny=16, p=2, g=2, ip=True, source=True, perturb=0.05, seed=4321, ns_flux=2)
    r_or = ob.residual(ob.oracle(), spec.oracle_problem(), spec.coords(), u.cpu().numpy())
    assert np.linalg.norm(r_or) <= 2e-10
