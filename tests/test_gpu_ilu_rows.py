"""The row-pipelined block-ILU(0) apply (one CTA per grid row) against the
data-flow apply on the same factors: both compute the same triangular solves
in different summation orders, so they agree to 1e-12 of the result's size in
FP64 and to 1e-5 with the FP32 factors."""
import numpy as np
import pytest
import torch

from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

CASES = [
    dict(pde=BURGERS, nx=7, ny=5, p=2),            # 9 x 9 blocks
    dict(pde=BURGERS, nx=4, ny=6, p=1, g=1),       # 4 x 4
    dict(pde=BURGERS, nx=5, ny=3, p=4),            # 25 x 25
    dict(pde=BURGERS, nx=1, ny=6, p=3),            # one column: no left neighbours
    dict(pde=BURGERS, nx=6, ny=1, p=3),            # one row: no waits between CTAs
    dict(pde=BURGERS, nx=1, ny=1, p=2),
    dict(pde=NS, nx=6, ny=4, p=2, ip=True),        # 36 x 36
    dict(pde=NS, nx=3, ny=5, p=3, ip=True),        # 64 x 64
]


@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_row_pipelined_apply_matches_data_flow_apply(kw, precision, tol):
    spec = Spec(**kw)
    ctx = spec.context()
    rng = np.random.default_rng(3)
    u = torch.from_numpy(spec.state(rng)).cuda()
    L = ctx.layout
    bs = L.block_size
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    res = torch.empty_like(u)
    ctx.form_jacobian_fd(u, res, vals)
    for trial in range(2):  # a second apply reuses the completion counters
        x = torch.from_numpy(rng.standard_normal(L.n_dof)).cuda()
        y_flow, y_rows = torch.empty_like(x), torch.empty_like(x)
        ctx.ilu_apply(vals, x, y_flow, precision, 1)
        ctx.ilu_apply(vals, x, y_rows, precision, 2, repeat=2)
        torch.cuda.synchronize()
        scale = float(y_flow.abs().max())
        assert float((y_rows - y_flow).abs().max()) <= tol * scale
