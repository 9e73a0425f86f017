"""Seeded synthetic workloads of the benchmark shapes (the reference publishes
no datasets for this path; every input here is generated from fixed seeds).

  burgers_config   - 2D viscous Burgers on [0,1]^2, nx x ny quads, p = 2 with
                     geometry order 2 (4x4 volume / 4-point face Gauss-Legendre),
                     mu = 1e-2, nonlinear advection b = (1, 0.5), Dirichlet u = 0,
                     u0 = sin(2 pi x) sin(2 pi y) at the Lagrange nodes + N(0, 1e-3).
  ns_mms_config    - 2D compressible Navier-Stokes manufactured solution on
                     [0,1]^2, p = 3, geometry order 2 (5x5 / 5-point rules),
                     gamma 1.4, Pr 0.72, mu = 1/Re = 0.01, Mach 0.3 pressure
                     level, Van Leer convective flux with interior penalty,
                     nodes perturbed by a seeded smooth displacement of
                     amplitude 0.05 h that keeps the domain boundary.
  batched_problems - independent 2D advection-diffusion problems of uneven
                     size and order: n x n quads with n uniform in [8, 96],
                     p uniform in {1, 2, 3, 4}, geometry order 1, viscosity
                     log-uniform in [1e-4, 1e-1], advection a = (cos t, sin t)
                     with t uniform in [0, 2 pi), Dirichlet data 1 left of the
                     line x = 0.5 + 0.3 y and 0 right of it (a boundary layer
                     and an interior front), seeded sinusoidal initial state;
                     grouped by p into batches.
"""
import ctypes as C

import numpy as np

from . import DIRICHLET, EXTRAPOLATION, FLUX_VANLEER, Context, workload_fn


def lattice_coords(nelem, geo_order, xmin=(0.0, 0.0), xmax=(1.0, 1.0)):
    """equispaced geometry-node lattice, x fastest, [n_nodes, 2]"""
    g = geo_order
    nnx, nny = nelem[0] * g + 1, nelem[1] * g + 1
    ix, iy = np.meshgrid(np.arange(nnx), np.arange(nny))
    x = xmin[0] + (xmax[0] - xmin[0]) * ix.ravel() / (nelem[0] * g)
    y = xmin[1] + (xmax[1] - xmin[1]) * iy.ravel() / (nelem[1] * g)
    return np.ascontiguousarray(np.stack([x, y], axis=1))


def perturb_smooth(coord, nelem, amp_frac, seed, xmin=(0.0, 0.0), xmax=(1.0, 1.0)):
    """seeded smooth displacement of every node, zero on the domain boundary:
    d_i = amp_frac h_i sin(pi xs) sin(pi ys) sin(2 pi (k_i . xs) + phase_i)"""
    rng = np.random.default_rng(seed)
    h = [(xmax[d] - xmin[d]) / nelem[d] for d in range(2)]
    xs = (coord[:, 0] - xmin[0]) / (xmax[0] - xmin[0])
    ys = (coord[:, 1] - xmin[1]) / (xmax[1] - xmin[1])
    bump = np.sin(np.pi * xs) * np.sin(np.pi * ys)
    k = rng.integers(1, 4, size=(2, 2))
    ph = rng.uniform(0, 2 * np.pi, size=2)
    out = coord.copy()
    for d in range(2):
        out[:, d] += amp_frac * h[d] * bump * np.sin(2 * np.pi * (k[d, 0] * xs + k[d, 1] * ys) + ph[d])
    return np.ascontiguousarray(out)


class Workload:
    """a configured Context plus the arrays that define its input state"""

    def __init__(self, ctx, coords, u0, params, name, keep):
        self.ctx, self.coords, self.u0, self.params, self.name = ctx, coords, u0, params, name
        self._keep = keep


def burgers_config(nx=32, ny=32, p=2, geo_order=2, seed=1234, device=0, interior_penalty=False,
                   perturb=0.0, mu=1e-2, b=(1.0, 0.5)):
    ctx = Context(device)
    ctx.mesh_uniform((nx, ny), (0.0, 0.0), (1.0, 1.0), geo_order, (DIRICHLET,) * 4, (0,) * 4)
    coords = lattice_coords((nx, ny), geo_order)
    if perturb:
        coords = perturb_smooth(coords, (nx, ny), perturb, seed)
    ctx.set_coords(coords)
    ctx.fespace(p)
    ctx.disc_burgers(mu, (0.0, 0.0), b)
    ctx.disc_options(interior_penalty, 0.0)
    zero = (C.c_double * 2)(1.0, 0.0)
    ctx.dirichlet(0, workload_fn("constant"), C.cast(zero, C.c_void_p))
    ctx.setup()
    xy = ctx.basis_node_coords()
    rng = np.random.default_rng(seed)
    u0 = np.sin(2 * np.pi * xy[..., 0]) * np.sin(2 * np.pi * xy[..., 1])
    u0 = u0.reshape(-1) + rng.normal(0.0, 1e-3, size=u0.size)
    return Workload(ctx, coords, np.ascontiguousarray(u0), dict(mu=mu, b=b, p=p, g=geo_order), "burgers", [zero])


def ns_mms_params(gamma=1.4, Pr=0.72, mu=0.01, mach=0.3, A=0.1, u0=1.0, v0=0.5):
    pinf = 1.0 * (u0 * u0 + v0 * v0) / (gamma * mach * mach)
    return (C.c_double * 7)(gamma, Pr, mu, pinf, A, u0, v0)


def ns_mms_config(nx=128, ny=128, p=3, geo_order=2, seed=4321, device=0, perturb=0.05, interior_penalty=True,
                  state_noise=1e-3, mu=0.01, conv_flux=FLUX_VANLEER):
    prm = ns_mms_params(mu=mu)
    ctx = Context(device)
    ctx.mesh_uniform((nx, ny), (0.0, 0.0), (1.0, 1.0), geo_order, (DIRICHLET,) * 4, (0,) * 4)
    coords = lattice_coords((nx, ny), geo_order)
    if perturb:
        coords = perturb_smooth(coords, (nx, ny), perturb, seed)
    ctx.set_coords(coords)
    ctx.fespace(p)
    ctx.disc_navier_stokes(prm[0], prm[1], prm[2], conv_flux)
    ctx.disc_options(interior_penalty, 0.0)
    user = C.cast(prm, C.c_void_p)
    ctx.dirichlet(0, workload_fn("ns_mms_state"), user)
    ctx.source(workload_fn("ns_mms_source"), user)
    ctx.setup()
    xy = ctx.basis_node_coords().reshape(-1, 2)
    st = np.zeros((xy.shape[0], 4))
    f = workload_fn("ns_mms_state")
    out = (C.c_double * 4)()
    pt = (C.c_double * 2)()
    for k in range(xy.shape[0]):
        pt[0], pt[1] = xy[k, 0], xy[k, 1]
        f(pt, out, user)
        st[k] = out[:]
    rng = np.random.default_rng(seed)
    st *= 1.0 + state_noise * rng.standard_normal(st.shape)
    return Workload(ctx, coords, np.ascontiguousarray(st.reshape(-1)),
                    dict(prm=list(prm), p=p, g=geo_order, conv_flux=conv_flux), "ns_mms", [prm])


def ns_mms_strip_config(plan, p=3, geo_order=2, seed=4321, device=0, perturb=0.05, interior_penalty=True,
                        state_noise=1e-3, mu=0.01):
    """one rank's part of the Navier-Stokes manufactured solution on the
    plan.nx x plan.ny mesh of square elements over [0, 1] x [0, ny / nx]
    (the single-rank workload is the whole of it, [0, 1]^2 when ny = nx):
    the sub-mesh of element rows [g0, g1) (iceicle_b200.partition) on the
    global perturbed nodes, with the state of ns_mms_config at its nodes
    (noise seeded by seed + rank)"""
    from .partition import sub_coords
    nx, ny, g = plan.nx, plan.ny, geo_order
    ymax = ny / nx
    coords = lattice_coords((nx, ny), g, (0.0, 0.0), (1.0, ymax))
    if perturb:
        coords = perturb_smooth(coords, (nx, ny), perturb, seed, (0.0, 0.0), (1.0, ymax))
    sub = sub_coords(plan, coords)
    prm = ns_mms_params(mu=mu)
    ctx = Context(device)
    h = ymax / ny
    ctx.mesh_uniform((nx, plan.rows), (0.0, plan.g0 * h), (1.0, plan.g1 * h), g, (DIRICHLET,) * 4, (0,) * 4)
    ctx.set_coords(sub)
    ctx.fespace(p)
    ctx.disc_navier_stokes(prm[0], prm[1], prm[2], FLUX_VANLEER)
    ctx.disc_options(interior_penalty, 0.0)
    user = C.cast(prm, C.c_void_p)
    ctx.dirichlet(0, workload_fn("ns_mms_state"), user)
    ctx.source(workload_fn("ns_mms_source"), user)
    ctx.setup()
    xy = ctx.basis_node_coords().reshape(-1, 2)
    st = np.zeros((xy.shape[0], 4))
    f = workload_fn("ns_mms_state")
    out = (C.c_double * 4)()
    pt = (C.c_double * 2)()
    for k in range(xy.shape[0]):
        pt[0], pt[1] = xy[k, 0], xy[k, 1]
        f(pt, out, user)
        st[k] = out[:]
    rng = np.random.default_rng(seed + plan.rank)
    st *= 1.0 + state_noise * rng.standard_normal(st.shape)
    return Workload(ctx, sub, np.ascontiguousarray(st.reshape(-1)),
                    dict(prm=list(prm), p=p, g=geo_order, rows=(plan.g0, plan.g1)), "ns_mms_strip", [prm])


def batched_problem_specs(n_problems=512, seed=2024, n_range=(8, 96), orders=(1, 2, 3, 4)):
    """the seeded problem list: dicts with n, p, mu, theta and the initial
    state's wave numbers and phases"""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_problems):
        out.append(dict(n=int(rng.integers(n_range[0], n_range[1] + 1)), p=int(rng.choice(orders)),
                        mu=float(10.0 ** rng.uniform(-4.0, -1.0)), theta=float(rng.uniform(0.0, 2 * np.pi)),
                        kx=int(rng.integers(1, 4)), ky=int(rng.integers(1, 4)),
                        phx=float(rng.uniform(0.0, 2 * np.pi)), phy=float(rng.uniform(0.0, 2 * np.pi))))
    return out


def advection_diffusion_problem(spec, device=0):
    """one problem of the list as a set-up Context and its initial state"""
    n, p = spec["n"], spec["p"]
    ctx = Context(device)
    ctx.mesh_uniform((n, n), (0.0, 0.0), (1.0, 1.0), 1, (DIRICHLET,) * 4, (0,) * 4)
    ctx.set_coords(lattice_coords((n, n), 1))
    ctx.fespace(p)
    a = (np.cos(spec["theta"]), np.sin(spec["theta"]))
    ctx.disc_burgers(spec["mu"], a, (0.0, 0.0))
    ctx.disc_options(False, 0.0)
    step = (C.c_double * 4)(0.5, 0.3, 1.0, 0.0)
    ctx.dirichlet(0, workload_fn("oblique_step"), C.cast(step, C.c_void_p))
    ctx.setup()
    ctx._keep.append(step)
    xy = ctx.basis_node_coords()
    u0 = np.sin(2 * np.pi * spec["kx"] * xy[..., 0] + spec["phx"]) * np.sin(2 * np.pi * spec["ky"] * xy[..., 1] +
                                                                           spec["phy"])
    return ctx, np.ascontiguousarray(u0.reshape(-1))


def batched_problems(n_problems=512, seed=2024, device=0):
    """the problem list grouped by basis order: {p: (batch Context, parts,
    concatenated initial state, [specs])}"""
    from . import batch
    specs = batched_problem_specs(n_problems, seed)
    groups = {}
    for sp in specs:
        groups.setdefault(sp["p"], []).append(sp)
    out = {}
    for p, lst in sorted(groups.items()):
        parts, states = [], []
        for sp in lst:
            c, u0 = advection_diffusion_problem(sp, device)
            parts.append(c)
            states.append(u0)
        out[p] = (batch(parts, device), parts, np.concatenate(states), lst)
    return out


def jitter_interior(coord, nelem, frac, seed):
    """seeded uniform displacement in [-frac h, frac h] of every interior node
    of a geometry-order-1 lattice (boundary nodes keep their place)"""
    rng = np.random.default_rng(seed)
    out = coord.copy()
    nx, ny = nelem
    h = (1.0 / nx, 1.0 / ny)
    for k in range(out.shape[0]):
        ix, iy = k % (nx + 1), k // (nx + 1)
        d = rng.uniform(-frac, frac, 2)
        if 0 < ix < nx and 0 < iy < ny:
            out[k, 0] += d[0] * h[0]
            out[k, 1] += d[1] * h[1]
    return np.ascontiguousarray(out)


def mdg_ice_config(n=64, p=1, seed=99, device=0, jitter=0.2):
    """MDG-ICE steady inviscid Burgers with an oblique discontinuity: n x n
    quads on [0, 1]^2, geometry order 1, (u^2 / 2)_x + u_y = 0 (a = (0, 1),
    b = (1, 0), mu = 0), u = 1 left of x = 0.4 + 0.2 y and -0.5 right of it;
    left, bottom and right Dirichlet with that state, top extrapolation;
    interior nodes jittered by a seeded +-0.2 h; every interior trace
    selected (geometry unknowns: their nodes, boundary nodes sliding along
    the box). Returns (workload, traces, x0)."""
    ctx = Context(device)
    ctx.mesh_uniform((n, n), (0.0, 0.0), (1.0, 1.0), 1, (DIRICHLET, DIRICHLET, DIRICHLET, EXTRAPOLATION), (0,) * 4)
    coords = jitter_interior(lattice_coords((n, n), 1), (n, n), jitter, seed)
    ctx.set_coords(coords)
    ctx.fespace(p)
    ctx.disc_burgers(0.0, (0.0, 1.0), (1.0, 0.0))
    ctx.disc_options(False, 0.0)
    step = (C.c_double * 4)(0.4, 0.2, 1.0, -0.5)
    ctx.dirichlet(0, workload_fn("oblique_step"), C.cast(step, C.c_void_p))
    ctx.setup()
    _, _, nint = ctx.topology()
    traces = np.arange(nint)
    ctx.mdg_select(traces, True)
    xy = ctx.basis_node_coords().reshape(-1, 2)
    u0 = np.where(xy[:, 0] < 0.4 + 0.2 * xy[:, 1], 1.0, -0.5)
    return Workload(ctx, coords, np.ascontiguousarray(u0), dict(n=n, p=p, jitter=jitter), "mdg_ice", [step]), \
        traces, ctx.mdg_get_x()
