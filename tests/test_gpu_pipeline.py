"""Residuals of host-resident states through the overlapped copy pipeline
(icx_form_residuals_host) against the device entry point: the same kernels,
so every residual is bit-identical, whatever the number of states and
whether the host memory is page-locked."""
import numpy as np
import pytest
import torch

from specs import NS, Spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_states,pinned", [(1, True), (5, True), (4, False)])
def test_host_pipeline_matches_device_residuals(n_states, pinned):
    spec = Spec(pde=NS, nx=5, ny=4, p=3, ip=True, source=True)
    ctx = spec.context()
    rng = np.random.default_rng(n_states)
    states = np.stack([spec.state(rng) for _ in range(n_states)])
    h_u = torch.from_numpy(states)
    h_r = torch.full_like(h_u, float("nan"))
    if pinned:
        h_u, h_r = h_u.pin_memory(), h_r.pin_memory()
    ms = ctx.form_residuals_host(h_u, h_r)
    assert ms > 0.0
    for k in range(n_states):
        du = torch.from_numpy(states[k]).cuda()
        dr = torch.empty_like(du)
        ctx.form_residual(du, dr)
        torch.cuda.synchronize()
        assert torch.equal(dr.cpu(), h_r[k])
