"""FP32 flux quadrature in the FD Jacobian (icx_form_jacobian_fd_f32) and
Newton as FP64 iterative refinement around it (icx_newton_options.precision 2).

* The FP32 blocks against the oracle's FP64 FD Jacobian: max |J32 - J| within
  2e-2 of max |J|. A one-sided FP32 difference with eps = sqrt(FLT_EPSILON)
  carries a rounding error of about FLT_EPSILON |F| / eps = 3.5e-4 |F| per
  entry, and the Navier-Stokes fluxes are an order of magnitude above the
  Jacobian entries (the pressure is ~1 / (gamma M^2) ~ 10 at Mach 0.3):
  about 1e-2 of the largest entry (measured 7e-3 to 9e-3; the Burgers
  cases below 2e-3). The residual the call writes is the FP64 residual bit
  for bit.
* Newton with FP32 linearisations converges to the FP64 Newton's state within
  1e-10 of the L2 norm of the larger of that state and the initial state: the
  outer residual, norm, line search and update are FP64, so only the
  iteration count can change.
"""
import numpy as np
import pytest
import torch

import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

CASES = [
    dict(pde=BURGERS, nx=6, ny=5, p=2),
    dict(pde=BURGERS, nx=5, ny=4, p=3, g=2),
    dict(pde=NS, nx=5, ny=4, p=2, ip=True),
    dict(pde=NS, nx=4, ny=4, p=3, g=2, ip=True, source=True),
]


@pytest.mark.parametrize("kw", CASES, ids=[str(i) for i in range(len(CASES))])
def test_fp32_blocks_against_oracle(kw):
    spec = Spec(**kw)
    ctx = spec.context()
    L = ctx.layout
    bs = L.block_size
    rng = np.random.default_rng(11)
    u0 = spec.state(rng)
    u = torch.from_numpy(u0).cuda()
    res32, res64 = torch.empty_like(u), torch.empty_like(u)
    v32 = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float32, device="cuda")
    v64 = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    ctx.form_jacobian_fd_f32(u, res32, v32)
    ctx.form_jacobian_fd(u, res64, v64)
    torch.cuda.synchronize()
    assert torch.equal(res32.view(torch.int64), res64.view(torch.int64))
    r_or, rowptr, colidx, v_or = ob.jacobian_bsr(spec.oracle_problem(), spec.coords(), u0)
    rp, ci = ctx.jacobian_pattern()
    assert np.array_equal(rp, rowptr) and np.array_equal(ci, colidx)
    j32 = v32.cpu().numpy().astype(np.float64).reshape(v_or.shape)
    err = np.abs(j32 - v_or).max() / np.abs(v_or).max()
    assert err <= 2e-2, err
    ctx.close()


@pytest.mark.parametrize("pde", ["burgers", "ns"])
def test_newton_fp32_quadrature_reaches_fp64_state(pde):
    import iceicle_b200 as ib
    from iceicle_b200.workloads import burgers_config, ns_mms_config
    wl = burgers_config(nx=16, ny=16) if pde == "burgers" else ns_mms_config(nx=12, ny=12, p=2, geo_order=2)
    out = {}
    # Burgers: to 1e-13, so that both states are within roundoff of the root
    # (its Jacobian's inverse amplifies a 1e-10 residual to ~1e-8 in the state)
    tau = 1e-13 if pde == "burgers" else 1e-10
    for prec in (0, 2):
        o = ib.default_newton_options()
        o.precision, o.gmres_rtol, o.tau_abs, o.kmax = prec, 1e-10, tau, 30
        u = torch.from_numpy(wl.u0.copy()).cuda()
        rep = wl.ctx.newton_solve(u, o)
        assert rep.converged, (prec, list(rep.residual_history[:rep.iterations + 1]))
        out[prec] = (u.cpu().numpy(), rep.iterations)
    a, b = out[0][0], out[2][0]
    # against the initial state's norm: the Burgers steady state is u = 0
    scale = max(np.linalg.norm(a), np.linalg.norm(wl.u0))
    assert np.linalg.norm(a - b) <= 1e-10 * scale, np.linalg.norm(a - b) / scale
