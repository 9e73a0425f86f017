"""Spacetime slabs (Burgers in (x, t)) coupled through SPACETIME_PAST faces:
marching two slabs, each solved on its own with the second taking the first's
top trace, gives the solution of the double-height slab solved at once (its
interior faces at the slab interface see the same time-upwind flux, and the
diffusive normal flux vanishes there since there is no diffusion along t)."""
import ctypes as C

import numpy as np
import pytest
import torch

import iceicle_b200 as ib

pytestmark = pytest.mark.gpu

STEP = (C.c_double * 4)(0.4, -0.1, 1.0, 0.25)  # u = 1 left of x = 0.4 - 0.1 t, 0.25 right of it


def _slab(nx, ny, t0, t1, bottom, p=2):
    ctx = ib.Context(0)
    ctx.mesh_uniform((nx, ny), (0.0, t0), (1.0, t1), 1,
                     (ib.DIRICHLET, bottom, ib.EXTRAPOLATION, ib.SPACETIME_FUTURE), (0, 0, 0, 0))
    ctx.fespace(p)
    ctx.disc_spacetime_burgers(5e-2, 0.3, 1.0)
    ctx.dirichlet(0, ib.workload_fn("oblique_step"), C.cast(STEP, C.c_void_p))
    ctx.setup()
    return ctx


def _solve(ctx, n):
    u = torch.full((n,), 0.5, dtype=torch.float64, device="cuda")
    o = ib.default_newton_options()
    o.tau_abs, o.kmax, o.gmres_rtol, o.gmres_max_it = 1e-12, 30, 1e-12, 5000
    rep = ctx.newton_solve(u, o)
    assert rep.converged, list(rep.residual_history[:rep.iterations + 1])
    return u


def test_two_coupled_slabs_equal_one_double_slab():
    nx, p = 8, 2
    nb = (p + 1) ** 2
    full = _slab(nx, 4, 0.0, 2.0, ib.DIRICHLET, p)
    u_full = _solve(full, nx * 4 * nb).cpu().numpy().reshape(4, nx, nb)
    s1 = _slab(nx, 2, 0.0, 1.0, ib.DIRICHLET, p)
    u1 = _solve(s1, nx * 2 * nb)
    s2 = _slab(nx, 2, 1.0, 2.0, ib.SPACETIME_PAST, p)
    s2.spacetime_connect(s1, u1)
    u2 = _solve(s2, nx * 2 * nb)
    a = np.concatenate([u1.cpu().numpy().reshape(2, nx, nb), u2.cpu().numpy().reshape(2, nx, nb)])
    assert np.linalg.norm(a - u_full) <= 1e-10 * np.linalg.norm(u_full)
    # the past trace matters: the unconnected second slab (no inflow in time) differs
    s3 = _slab(nx, 2, 1.0, 2.0, ib.SPACETIME_PAST, p)
    r = torch.empty_like(u2)
    s3.form_residual(u2, r)
    torch.cuda.synchronize()
    assert float(torch.linalg.vector_norm(r)) > 1e-3


def test_connection_errors():
    s1 = _slab(4, 2, 0.0, 1.0, ib.DIRICHLET)
    u1 = torch.zeros(4 * 2 * 9, dtype=torch.float64, device="cuda")
    with pytest.raises(ib.IcxError):
        s1.spacetime_connect(s1, u1)  # no SPACETIME_PAST faces
    far = _slab(4, 2, 1.5, 2.5, ib.SPACETIME_PAST)
    with pytest.raises(ib.IcxError):
        far.spacetime_connect(s1, u1)  # slabs do not meet
