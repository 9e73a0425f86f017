"""Problem specifications shared by the oracle side (orc_problem) and the GPU
side (icx Context), so both evaluate exactly the same discretization on the
same mesh coordinates and state. Test infrastructure only.

The oracle side takes everything from the oracle library: mesh coordinates
(oracle_bindings), boundary data and sources (its own orc_wl_* callbacks)
and basis-node coordinates. Nothing here loads the product library unless
a GPU context is asked for (Spec.context)."""
import ctypes as C

import numpy as np

import oracle_bindings as ob

BURGERS, NS = 0, 1


def ns_mms_params(gamma=1.4, Pr=0.72, mu=0.01, mach=0.3, A=0.1, u0=1.0, v0=0.5):
    """{gamma, Pr, mu, pinf, A, u0, v0} of the manufactured Navier-Stokes
    solution, pinf = rho_inf |u_inf|^2 / (gamma M^2)"""
    pinf = 1.0 * (u0 * u0 + v0 * v0) / (gamma * mach * mach)
    return (C.c_double * 7)(gamma, Pr, mu, pinf, A, u0, v0)


class Spec:
    def __init__(self, pde=BURGERS, nx=4, ny=3, g=2, p=2, bct=(3, 3, 3, 3), bcf=(0, 0, 0, 0), ip=False,
                 sigma_ic=0.0, mu=0.01, a=(0.3, -0.2), b=(1.0, 0.5), perturb=0.1, seed=7,
                 dirichlet=None, neumann=None, source=False, spacetime=False, basis=0, ns_flux=1, ns_mu=0.01,
                 walls=(), free_stream=None, sutherland=None):
        self.pde, self.nx, self.ny, self.g, self.p = pde, nx, ny, g, p
        self.bct, self.bcf, self.ip, self.sigma_ic = tuple(bct), tuple(bcf), ip, sigma_ic
        self.spacetime = spacetime
        self.basis = basis
        # Navier-Stokes: convective flux (1 Van Leer, 2 Roe), viscosity, wall
        # temperatures per bcflag, free stream (rho, |u|, (dx, dy), T)
        self.ns_flux, self.ns_mu, self.walls = ns_flux, ns_mu, tuple(walls)
        self.free_stream = free_stream
        # DimensionlessSutherlands ratios (mu_0/ref.mu, T_0/ref.T, T_s/ref.T), or constant viscosity
        self.sutherland = sutherland
        if spacetime:  # Burgers in (x, t): the time component of the flux is u
            a, b = (a[0], 1.0), (b[0], 0.0)
        self.mu, self.a, self.b = mu, a, b
        self.perturb, self.seed = perturb, seed
        self.neq = 1 if pde == BURGERS else 4
        # boundary data: list of (function name, params) per flag
        if dirichlet is None:
            dirichlet = [("constant", [1, 0.25])] if pde == BURGERS else [("ns_mms_state", None)]
        if neumann is None:
            neumann = [("constant", [1, 0.1])] if pde == BURGERS else [("constant", [4, 0.0, 0.0, 0.0, 0.0])]
        self.dirichlet, self.neumann, self.source = dirichlet, neumann, source
        self._keep = []

    @property
    def E(self):
        return self.nx * self.ny

    @property
    def nb(self):
        return (self.p + 1) ** 2

    @property
    def N(self):
        return self.E * self.nb * self.neq

    def _geometry_problem(self):
        pb = ob.Problem()
        pb.nx, pb.ny, pb.geo_order, pb.p = self.nx, self.ny, self.g, self.p
        pb.xmin[:] = [0.0, 0.0]
        pb.xmax[:] = [1.0, 1.0]
        return pb

    def coords(self):
        """geometry nodes: the equispaced lattice plus the seeded smooth
        perturbation (oracle-side copy of the workload definition)"""
        pb = self._geometry_problem()
        c = ob.lattice_coords(pb)
        if self.perturb:
            c = ob.perturb_smooth(pb, c, self.perturb, self.seed)
        return c

    def _params(self, name, prm):
        if name.startswith("ns_mms"):
            arr = ns_mms_params(mu=self.ns_mu)
        else:
            arr = (C.c_double * len(prm))(*prm)
        self._keep.append(arr)
        return arr

    def fn(self, name):
        """C function pointer of the oracle's workload callback orc_wl_<name>"""
        return C.cast(getattr(ob.oracle().lib, "orc_wl_" + name), ob.POINT_FN)

    def mms_state(self, coords, seed=4321, noise=1e-3):
        """the Navier-Stokes workload's initial state: the manufactured state at
        the Lagrange basis nodes times (1 + noise N(0, 1)), seeded like the
        product's workload builder"""
        pb = self._geometry_problem()
        xy = ob.basis_node_coords(pb, coords).reshape(-1, 2)
        prm = ns_mms_params(mu=self.ns_mu)
        f = self.fn("ns_mms_state")
        st = np.zeros((xy.shape[0], 4))
        out = (C.c_double * 4)()
        pt = (C.c_double * 2)()
        for k in range(xy.shape[0]):
            pt[0], pt[1] = xy[k, 0], xy[k, 1]
            f(pt, out, C.cast(prm, C.c_void_p))
            st[k] = out[:]
        rng = np.random.default_rng(seed)
        st *= 1.0 + noise * rng.standard_normal(st.shape)
        return np.ascontiguousarray(st.reshape(-1))

    def state(self, rng):
        if self.pde == BURGERS:
            return 0.3 * rng.standard_normal(self.N)
        base = np.tile([1.0, 0.5, 0.2, 3.0], self.N // 4)
        return base * (1.0 + 0.05 * rng.standard_normal(self.N))

    def oracle_problem(self):
        pb = ob.Problem()
        pb.pde, pb.nx, pb.ny, pb.geo_order, pb.p = self.pde, self.nx, self.ny, self.g, self.p
        pb.xmin[:] = [0.0, 0.0]
        pb.xmax[:] = [1.0, 1.0]
        pb.bctype[:] = list(self.bct)
        pb.bcflag[:] = list(self.bcf)
        pb.interior_penalty = int(self.ip)
        pb.sigma_ic = self.sigma_ic
        pb.mu = self.mu
        pb.a[:] = list(self.a)
        pb.b[:] = list(self.b)
        pb.spacetime = int(self.spacetime)
        pb.basis = int(self.basis)
        pb.gamma, pb.Pr, pb.ns_mu = 1.4, 0.72, self.ns_mu
        pb.ns_flux = self.ns_flux
        if self.sutherland is not None:
            pb.ns_visc = 1
            pb.suth[:] = list(self.sutherland)
        pb.n_wall = len(self.walls)
        for i, t in enumerate(self.walls):
            pb.wall_T[i] = t
        if self.free_stream is not None:
            pb.fs_rho, pb.fs_u_inf, (pb.fs_dir[0], pb.fs_dir[1]), pb.fs_T = self.free_stream
        pb.n_dirichlet = len(self.dirichlet)
        for i, (name, prm) in enumerate(self.dirichlet):
            arr = self._params(name, prm)
            pb.dirichlet[i] = C.cast(self.fn(name), ob.POINT_FN)
            pb.dirichlet_user[i] = C.cast(arr, C.c_void_p)
        pb.n_neumann = len(self.neumann)
        for i, (name, prm) in enumerate(self.neumann):
            arr = self._params(name, prm)
            pb.neumann[i] = C.cast(self.fn(name), ob.POINT_FN)
            pb.neumann_user[i] = C.cast(arr, C.c_void_p)
        if self.source:
            arr = self._params("ns_mms_source", None)
            pb.source = C.cast(self.fn("ns_mms_source"), ob.POINT_FN)
            pb.source_user = C.cast(arr, C.c_void_p)
        return pb

    def context(self, coords=None):
        """the same problem as a GPU context; boundary data and sources are the
        product's own exported callbacks (icx_wl_*), so the parity tests also
        check them against the oracle's"""
        import iceicle_b200 as ib
        ctx = ib.Context(0)
        ctx.mesh_uniform((self.nx, self.ny), (0.0, 0.0), (1.0, 1.0), self.g, self.bct, self.bcf)
        ctx.set_coords(self.coords() if coords is None else coords)
        ctx.fespace(self.p, self.basis)
        if self.pde == BURGERS and self.spacetime:
            ctx.disc_spacetime_burgers(self.mu, self.a[0], self.b[0])
        elif self.pde == BURGERS:
            ctx.disc_burgers(self.mu, self.a, self.b)
        else:
            ctx.disc_navier_stokes(1.4, 0.72, self.ns_mu, self.ns_flux)
            if self.sutherland is not None:
                ctx.disc_ns_viscosity(1, *self.sutherland)
            if self.walls or self.free_stream is not None:
                fs = self.free_stream or (1.0, 0.0, (1.0, 0.0), 1.0)
                ctx.disc_ns_boundary(self.walls, fs[0], fs[1], fs[2], fs[3])
        ctx.disc_options(self.ip, self.sigma_ic)
        for i, (name, prm) in enumerate(self.dirichlet):
            ctx.dirichlet(i, ib.workload_fn(name), C.cast(self._params(name, prm), C.c_void_p))
        for i, (name, prm) in enumerate(self.neumann):
            ctx.neumann(i, ib.workload_fn(name), C.cast(self._params(name, prm), C.c_void_p))
        if self.source:
            ctx.source(ib.workload_fn("ns_mms_source"), C.cast(self._params("ns_mms_source", None), C.c_void_p))
        ctx.setup()
        return ctx
