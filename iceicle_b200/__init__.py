"""iceicle_b200: B200-native DG residual / FD-Jacobian / Newton path.

Python mirror of the reference interface for this path, over the C ABI in
include/iceicle_b200.h (libiceicle_b200.so, built in-tree for sm_100a):

  AbstractMesh.uniform(...)   <- AbstractMesh uniform constructor (mesh.hpp:553-913)
  FESpace(mesh, p)            <- FESpace (fespace.hpp:200-416)
  BurgersCoefficients / ConservationLawDDG.burgers(...) / .navier_stokes(...)
                              <- ConservationLawDDG + flux functors (conservation_law.hpp:92-218)
  form_residual(fespace, disc, u, res)           (form_residual.hpp:56-268)
  form_jacobian_fd(fespace, disc, u, res, vals)  (form_petsc_jacobian.hpp:55-317)
  NewtonSolver(fespace, disc, criteria, ls).solve(u)  (petsc_newton.hpp:37-337)

Device arrays are torch CUDA tensors (float64). There is no CPU fallback: a
missing or unloadable extension raises immediately.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libiceicle_b200.so")

POINT_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p)

# BOUNDARY_CONDITIONS values of the reference (geometry/face.hpp:23-90)
PERIODIC, PARALLEL_COM, NEUMANN, DIRICHLET, EXTRAPOLATION = 0, 1, 2, 3, 4
RIEMANN, NO_SLIP_ISOTHERMAL, SLIP_WALL, WALL_GENERAL = 5, 6, 7, 8
SPACETIME_PAST, SPACETIME_FUTURE = 11, 12
BASIS_LAGRANGE, BASIS_LEGENDRE = 0, 1
SPACETIME_FUTURE, INTERIOR = 12, 13
PDE_BURGERS, PDE_NAVIER_STOKES = 0, 1
FLUX_UPWIND, FLUX_VANLEER, FLUX_ROE = 0, 1, 2

STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "UNSUPPORTED", 4: "NONFINITE", 5: "NOT_CONVERGED",
          6: "NOMEM", 7: "SIZE", 8: "NO_DEVICE"}


class IcxError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"icx status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class LayoutInfo(C.Structure):
    _fields_ = [("n_elem", C.c_int), ("nbasis", C.c_int), ("neq", C.c_int), ("block_size", C.c_int),
                ("n_dof", C.c_longlong), ("n_faces", C.c_int), ("n_interior_faces", C.c_int),
                ("n_nodes", C.c_int), ("nnz_blocks", C.c_int), ("nq_vol", C.c_int), ("nq_face", C.c_int)]


class NewtonOptions(C.Structure):
    _fields_ = [("tau_abs", C.c_double), ("tau_rel", C.c_double), ("kmax", C.c_int),
                ("linesearch", C.c_int), ("ls_max_it", C.c_int), ("ls_alpha_initial", C.c_double),
                ("ls_alpha_max", C.c_double), ("ls_alpha_min", C.c_double), ("ls_c1", C.c_double),
                ("ls_c2", C.c_double), ("gmres_restart", C.c_int), ("gmres_max_it", C.c_int),
                ("gmres_rtol", C.c_double), ("preconditioner", C.c_int), ("verbosity", C.c_int),
                ("precision", C.c_int), ("pc_sweeps", C.c_int), ("cuda_graphs", C.c_int), ("ilu_tile", C.c_int),
                ("matrix_free", C.c_int), ("gmres_cgs_refine", C.c_int)]


class ExplicitOptions(C.Structure):
    _fields_ = [("scheme", C.c_int), ("timestep", C.c_int), ("dt", C.c_double), ("cfl", C.c_double),
                ("termination", C.c_int), ("ntime", C.c_int), ("tfinal", C.c_double)]


class ExplicitReport(C.Structure):
    _fields_ = [("steps", C.c_int), ("time", C.c_double), ("dt_last", C.c_double), ("lambda_max", C.c_double),
                ("singular_elements", C.c_int)]


class NewtonReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("r0", C.c_double), ("r_final", C.c_double),
                ("linear_iterations_total", C.c_int), ("residual_history", C.c_double * 64),
                ("alpha_history", C.c_double * 64), ("pc_fallbacks", C.c_int),
                ("linear_iterations", C.c_int * 64), ("graph_steps", C.c_int)]


class PsetStats(C.Structure):
    _fields_ = [("newton_rounds", C.c_int), ("arnoldi_steps", C.c_int), ("graph_launches", C.c_int),
                ("line_search_rounds", C.c_int), ("orders", C.c_int)]


class LpcTrainOptions(C.Structure):
    _fields_ = [("steps", C.c_int), ("batch", C.c_int), ("random", C.c_int), ("sweeps", C.c_int),
                ("lr", C.c_double), ("seed", C.c_ulonglong)]


class LpcTrainReport(C.Structure):
    _fields_ = [("steps", C.c_int), ("loss_first", C.c_double), ("loss_last", C.c_double),
                ("loss_history", C.c_double * 64)]


class TileChoice(C.Structure):
    """launch shapes of the tunable kernels (0: the compiled default)"""
    _fields_ = [("face_minb", C.c_int), ("vol_threads", C.c_int), ("vol_minb", C.c_int),
                ("ilu_rows", C.c_int * 2), ("ilu_ctas", C.c_int * 2), ("ilu_sched", C.c_int * 2)]

    def as_dict(self):
        return {"face_minb": self.face_minb, "vol_threads": self.vol_threads, "vol_minb": self.vol_minb,
                "ilu_rows": list(self.ilu_rows), "ilu_ctas": list(self.ilu_ctas),
                "ilu_sched": list(self.ilu_sched)}


class TuneReport(C.Structure):
    _fields_ = [("chosen", TileChoice), ("from_cache", C.c_int), ("n_timed", C.c_int), ("n_rejected", C.c_int),
                ("residual_ms_default", C.c_double), ("residual_ms_tuned", C.c_double),
                ("ilu_ms_default", C.c_double * 2), ("ilu_ms_tuned", C.c_double * 2)]


TUNE_RESIDUAL, TUNE_ILU, TUNE_ILU_FP32, TUNE_RETIME = 1, 2, 4, 8


_lib = None


def lib():
    """The loaded extension; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"iceicle_b200 CUDA extension not built: {LIB_PATH} (run iceicle_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        sig = {
            "icx_create": (C.c_int, [C.POINTER(vp), C.c_int]),
            "icx_destroy": (None, [vp]),
            "icx_last_error": (C.c_char_p, [vp]),
            "icx_mesh_uniform": (C.c_int, [vp, C.c_int, ip, dp, dp, C.c_int, ip, ip]),
            "icx_mesh_set_coords": (C.c_int, [vp, vp]),
            "icx_mesh_get_coords": (C.c_int, [vp, vp]),
            "icx_mesh_topology": (C.c_int, [vp, vp, vp, ip]),
            "icx_fespace": (C.c_int, [vp, C.c_int]),
            "icx_disc_burgers": (C.c_int, [vp, C.c_double, dp, dp]),
            "icx_disc_spacetime_burgers": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
            "icx_spacetime_connect": (C.c_int, [vp, vp, vp]),
            "icx_fespace_basis": (C.c_int, [vp, C.c_int, C.c_int]),
            "icx_form_residuals_host": (C.c_int, [vp, C.c_int, vp, vp, dp]),
            "icx_ilu_apply": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_int, C.c_int, dp]),
            "icx_disc_navier_stokes": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_int]),
            "icx_disc_ns_viscosity": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_double]),
            "icx_disc_ns_boundary": (C.c_int, [vp, dp, C.c_int, C.c_double, C.c_double, dp, C.c_double,
                                               C.c_double]),
            "icx_disc_options": (C.c_int, [vp, C.c_int, C.c_double]),
            "icx_disc_dirichlet": (C.c_int, [vp, C.c_int, POINT_FN, vp]),
            "icx_disc_neumann": (C.c_int, [vp, C.c_int, POINT_FN, vp]),
            "icx_disc_source": (C.c_int, [vp, POINT_FN, vp]),
            "icx_setup": (C.c_int, [vp]),
            "icx_get_layout": (C.c_int, [vp, C.POINTER(LayoutInfo)]),
            "icx_form_residual": (C.c_int, [vp, vp, vp, vp]),
            "icx_jacobian_pattern": (C.c_int, [vp, vp, vp]),
            "icx_form_jacobian_fd": (C.c_int, [vp, vp, vp, vp, C.c_double, vp]),
            "icx_form_jacobian_fd_f32": (C.c_int, [vp, vp, vp, vp, vp]),
            "icx_bsr_spmv": (C.c_int, [vp, vp, vp, vp, vp]),
            "icx_newton_default_options": (C.c_int, [C.POINTER(NewtonOptions)]),
            "icx_explicit_default_options": (C.c_int, [C.POINTER(ExplicitOptions)]),
            "icx_mfnk_solve": (C.c_int, [vp, vp, C.POINTER(NewtonOptions), C.POINTER(NewtonReport)]),
            "icx_batch_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.POINTER(vp)]),
            "icx_batch_offsets": (C.c_int, [vp, ip]),
            "icx_pset_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.POINTER(vp)]),
            "icx_pset_destroy": (None, [vp]),
            "icx_pset_offsets": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
            "icx_pset_residual": (C.c_int, [vp, vp, vp]),
            "icx_pset_newton_solve": (C.c_int, [vp, vp, C.POINTER(NewtonOptions), C.POINTER(NewtonReport),
                                                C.POINTER(PsetStats)]),
            "icx_pset_last_error": (C.c_char_p, [vp]),
            "icx_explicit_solve": (C.c_int, [vp, vp, C.POINTER(ExplicitOptions), C.POINTER(ExplicitReport)]),
            "icx_mass_inverse_apply": (C.c_int, [vp, vp, vp, vp]),
            "icx_newton_solve": (C.c_int, [vp, vp, C.POINTER(NewtonOptions), C.POINTER(NewtonReport)]),
            "icx_basis_node_coords": (C.c_int, [vp, vp]),
            "icx_krylov_samples": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                             vp, ip, ip, dp]),
            "icx_lpc_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_ulonglong]),
            "icx_lpc_destroy": (None, [vp]),
            "icx_lpc_info": (C.c_int, [vp, ip, ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
            "icx_lpc_get_params": (C.c_int, [vp, vp]),
            "icx_lpc_set_params": (C.c_int, [vp, vp]),
            "icx_lpc_attach": (C.c_int, [vp, vp]),
            "icx_lpc_forward": (C.c_int, [vp, vp, vp]),
            "icx_lpc_train": (C.c_int, [vp, vp, C.c_int, vp, C.POINTER(LpcTrainOptions), C.POINTER(LpcTrainReport)]),
            "icx_lpc_calibrate": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, dp]),
            "icx_write_restart": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_char_p]),
            "icx_read_restart": (C.c_int, [vp, vp, C.c_char_p, C.c_int, C.c_char_p]),
            "icx_write_vtu": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_char_p, C.c_char_p,
                                        C.POINTER(C.c_char_p), C.c_int]),
            "icx_write_vtu_mdg": (C.c_int, [vp, vp, C.c_int, C.c_char_p, C.c_char_p, C.POINTER(C.c_char_p),
                                            C.c_int]),
            "icx_form_residual_timed": (C.c_int, [vp, vp, vp, vp, dp, dp]),
            "icx_form_residual_noalloc": (C.c_int, [vp, vp, vp, vp]),
            "icx_gmres_solve": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_int, C.c_double, C.c_int, ip, dp, vp]),
            "icx_mdg_select": (C.c_int, [vp, C.c_int, vp, C.c_int]),
            "icx_mdg_info": (C.c_int, [vp, ip, ip]),
            "icx_mdg_selected_nodes": (C.c_int, [vp, vp]),
            "icx_mdg_get_x": (C.c_int, [vp, vp]),
            "icx_mdg_set_x": (C.c_int, [vp, vp]),
            "icx_form_mdg_residual": (C.c_int, [vp, vp, vp, vp]),
            "icx_form_residual_mdg": (C.c_int, [vp, vp, vp, vp, vp, vp]),
            "icx_mdg_jacobian_pattern": (C.c_int, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                                    C.POINTER(C.c_longlong), vp, vp]),
            "icx_form_jacobian_mdg_fd": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, vp]),
            "icx_autotune": (C.c_int, [vp, vp, C.c_int, C.POINTER(TuneReport)]),
            "icx_tile_get": (C.c_int, [vp, C.POINTER(TileChoice)]),
            "icx_tile_set": (C.c_int, [vp, C.POINTER(TileChoice)]),
            "icx_set_ilu_tile": (C.c_int, [vp, C.c_int]),
            "icx_gemm_bf16_nt": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, vp, C.c_int, vp,
                                           C.c_int, vp, C.c_int, C.c_int, C.c_int, vp]),
            "icx_get_ilu_tile": (C.c_int, [vp]),
            "icx_set_ilu_groups": (C.c_int, [vp, vp]),
            "icx_pc_factor": (C.c_int, [vp, vp, C.c_int]),
            "icx_pc_apply": (C.c_int, [vp, vp, vp, C.c_int, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(t):
    """raw pointer of a torch tensor or numpy array"""
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return t.ctypes.data_as(C.c_void_p)


def _stream_ptr(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


class Context:
    """One icx_ctx: mesh + finite element space + discretization on one device."""

    def __init__(self, device=0):
        self._h = C.c_void_p()
        self._keep = []  # callbacks must outlive the context
        st = lib().icx_create(C.byref(self._h), device)
        if st != 0:
            raise IcxError(st, "icx_create")

    def _check(self, st, what):
        if st != 0:
            msg = lib().icx_last_error(self._h)
            raise IcxError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self._h:
            lib().icx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- mesh / space / disc --------------------------------------------
    def mesh_uniform(self, nelem, xmin, xmax, geo_order, bctypes, bcflags):
        ne = (C.c_int * 2)(*nelem)
        a = (C.c_double * 2)(*xmin)
        b = (C.c_double * 2)(*xmax)
        bt = (C.c_int * 4)(*bctypes)
        bf = (C.c_int * 4)(*bcflags)
        self._check(lib().icx_mesh_uniform(self._h, 2, ne, a, b, geo_order, bt, bf), "mesh_uniform")
        self.nelem, self.geo_order = tuple(nelem), geo_order

    @property
    def n_nodes(self):
        g = self.geo_order
        return (self.nelem[0] * g + 1) * (self.nelem[1] * g + 1)

    def set_coords(self, xy):
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        assert xy.size == 2 * self.n_nodes
        self._check(lib().icx_mesh_set_coords(self._h, _ptr(xy)), "set_coords")

    def get_coords(self):
        xy = np.zeros((self.n_nodes, 2))
        self._check(lib().icx_mesh_get_coords(self._h, _ptr(xy)), "get_coords")
        return xy

    def topology(self):
        E = self.nelem[0] * self.nelem[1]
        ng = (self.geo_order + 1) ** 2
        nx, ny = self.nelem
        nf = (nx - 1) * ny + nx * (ny - 1) + 2 * nx + 2 * ny
        conn = np.zeros((E, ng), dtype=np.int32)
        faces = np.zeros((nf, 7), dtype=np.int32)
        ni = C.c_int()
        self._check(lib().icx_mesh_topology(self._h, _ptr(conn), _ptr(faces), C.byref(ni)), "topology")
        return conn, faces, ni.value

    def fespace(self, p, basis=0):
        """tensor-product space of order p: basis BASIS_LAGRANGE (0) or BASIS_LEGENDRE (1)"""
        if basis:
            self._check(lib().icx_fespace_basis(self._h, p, basis), "fespace")
        else:
            self._check(lib().icx_fespace(self._h, p), "fespace")
        self.p = p
        self.basis = basis

    def disc_spacetime_burgers(self, mu, a, b):
        """Burgers in (x, t): the second mesh coordinate is time"""
        self._check(lib().icx_disc_spacetime_burgers(self._h, mu, a, b), "disc_spacetime_burgers")

    def spacetime_connect(self, past, u_past):
        """take the solved slab `past` (state u_past, device) as the exterior
        state of this slab's SPACETIME_PAST faces"""
        self._check(lib().icx_spacetime_connect(self._h, past._h, _ptr(u_past)), "spacetime_connect")

    def disc_burgers(self, mu, a, b):
        self._check(lib().icx_disc_burgers(self._h, mu, (C.c_double * 2)(*a), (C.c_double * 2)(*b)), "disc_burgers")

    def disc_navier_stokes(self, gamma=1.4, Pr=0.72, mu=0.01, conv_flux=FLUX_VANLEER):
        self._check(lib().icx_disc_navier_stokes(self._h, gamma, Pr, mu, conv_flux), "disc_navier_stokes")

    def disc_ns_boundary(self, wall_temperatures=(), rho_inf=1.0, u_inf=0.0, u_direction=(1.0, 0.0), T_inf=1.0,
                         Rgas=287.052874):
        """Navier-Stokes wall temperatures (per bcflag) and free stream of the
        PDE-level boundaries (Physics::isothermal_temperatures / free_stream)"""
        tw = (C.c_double * 8)(*wall_temperatures)
        ud = (C.c_double * 2)(*u_direction)
        self._check(lib().icx_disc_ns_boundary(self._h, tw, len(wall_temperatures), rho_inf, u_inf, ud, T_inf, Rgas),
                    "disc_ns_boundary")

    def disc_ns_viscosity(self, kind=0, mu_ratio=0.0, T0_ratio=1.0, Ts_ratio=0.0):
        """Navier-Stokes viscosity law: 0 constant, 1 DimensionlessSutherlands
        with the ratios mu_0/ref.mu, T_0/ref.T, T_s/ref.T"""
        self._check(lib().icx_disc_ns_viscosity(self._h, int(kind), mu_ratio, T0_ratio, Ts_ratio), "disc_ns_viscosity")

    def disc_options(self, interior_penalty=False, sigma_ic=0.0):
        self._check(lib().icx_disc_options(self._h, int(interior_penalty), float(sigma_ic)), "disc_options")

    def _cb(self, fn):
        if isinstance(fn, POINT_FN):
            cb = fn
        elif isinstance(fn, C._CFuncPtr):
            cb = C.cast(fn, POINT_FN)
        else:
            cb = POINT_FN(fn)
        self._keep.append(cb)
        return cb

    def dirichlet(self, flag, fn, user=None):
        self._check(lib().icx_disc_dirichlet(self._h, flag, self._cb(fn), user), "dirichlet")

    def neumann(self, flag, fn, user=None):
        self._check(lib().icx_disc_neumann(self._h, flag, self._cb(fn), user), "neumann")

    def source(self, fn, user=None):
        self._check(lib().icx_disc_source(self._h, self._cb(fn), user), "source")

    def setup(self):
        self._check(lib().icx_setup(self._h), "setup")
        info = LayoutInfo()
        self._check(lib().icx_get_layout(self._h, C.byref(info)), "get_layout")
        self.layout = info
        return info

    # --- hot path ---------------------------------------------------------
    def basis_node_coords(self):
        """physical coordinates of each element's Lagrange nodes, [E, nbasis, 2]"""
        E = self.nelem[0] * self.nelem[1]
        nb = (self.p + 1) ** 2
        xy = np.zeros((E, nb, 2))
        self._check(lib().icx_basis_node_coords(self._h, _ptr(xy)), "basis_node_coords")
        return xy

    def form_residual(self, u, res, stream=None):
        self._check(lib().icx_form_residual(self._h, _ptr(u), _ptr(res), _stream_ptr(stream)), "form_residual")

    def ilu_apply(self, vals, x, y, precision=0, schedule=0, repeat=1):
        """y = M^-1 x with the block-ILU(0) factors of vals (schedule 0 or 1:
        the solvers' data-flow apply, 2: row-pipelined), applied `repeat`
        times after one factorization; returns the mean ms per apply"""
        ms = C.c_double()
        self._check(lib().icx_ilu_apply(self._h, _ptr(vals), _ptr(x), _ptr(y), precision, schedule, repeat,
                                        C.byref(ms)), "ilu_apply")
        return ms.value

    @property
    def ilu_tile(self):
        """side (in elements) of the tiles of the block-ILU(0) preconditioner; 0: the whole grid"""
        return lib().icx_get_ilu_tile(self._h)

    @ilu_tile.setter
    def ilu_tile(self, tile):
        self._check(lib().icx_set_ilu_tile(self._h, int(tile)), "set_ilu_tile")

    def set_ilu_groups(self, groups):
        """block-ILU(0) per element group (array of E ints), None: back to the tiling"""
        g = None if groups is None else np.ascontiguousarray(groups, dtype=np.int32)
        self._check(lib().icx_set_ilu_groups(self._h, _ptr(g) if g is not None else None), "set_ilu_groups")
        self._groups = g

    def pc_factor(self, vals, precision=0):
        """block-ILU(0) factors of the BSR values (the tiling / groups in force)"""
        self._check(lib().icx_pc_factor(self._h, _ptr(vals), precision), "pc_factor")

    def pc_apply(self, x, y, precision=0, stream=None):
        """y = M^-1 x with the factors of the last pc_factor"""
        self._check(lib().icx_pc_apply(self._h, _ptr(x), _ptr(y), precision, _stream_ptr(stream)), "pc_apply")

    def autotune(self, u, parts=TUNE_RESIDUAL | TUNE_ILU | TUNE_ILU_FP32):
        """times every compiled launch shape of the selected kernels at the
        device state u, keeps the fastest whose output is bit-identical to the
        default's, and returns the report as a dict"""
        rep = TuneReport()
        self._check(lib().icx_autotune(self._h, _ptr(u), parts, C.byref(rep)), "autotune")
        return {"chosen": rep.chosen.as_dict(), "from_cache": rep.from_cache, "n_timed": rep.n_timed,
                "n_rejected": rep.n_rejected, "residual_ms_default": rep.residual_ms_default,
                "residual_ms_tuned": rep.residual_ms_tuned, "ilu_ms_default": list(rep.ilu_ms_default),
                "ilu_ms_tuned": list(rep.ilu_ms_tuned)}

    @property
    def tile(self):
        """the context's launch shapes (dict of TileChoice fields)"""
        t = TileChoice()
        self._check(lib().icx_tile_get(self._h, C.byref(t)), "tile_get")
        return t.as_dict()

    @tile.setter
    def tile(self, d):
        t = TileChoice()
        d = dict(d)
        t.face_minb = d.get("face_minb", 0)
        t.vol_threads = d.get("vol_threads", 0)
        t.vol_minb = d.get("vol_minb", 0)
        for k, v in enumerate(d.get("ilu_rows", [0, 0])):
            t.ilu_rows[k] = v
        for k, v in enumerate(d.get("ilu_ctas", [0, 0])):
            t.ilu_ctas[k] = v
        for k, v in enumerate(d.get("ilu_sched", [0, 0])):
            t.ilu_sched[k] = v
        self._check(lib().icx_tile_set(self._h, C.byref(t)), "tile_set")

    def form_residuals_host(self, u, res):
        """residuals of the states u[k] (host arrays or CPU tensors, [n_states][n_dof],
        pinned for overlap) into res[k], with the copies of consecutive states
        overlapped; returns the device time in ms"""
        n = u.shape[0] if len(u.shape) > 1 else 1
        ms = C.c_double()
        self._check(lib().icx_form_residuals_host(self._h, n, _ptr(u), _ptr(res), C.byref(ms)),
                    "form_residuals_host")
        return ms.value

    def form_residual_noalloc(self, u, res, stream=None):
        """icx_form_residual_noalloc: same result, face scratch in a fixed
        device array instead of context memory; allocates nothing"""
        self._check(lib().icx_form_residual_noalloc(self._h, _ptr(u), _ptr(res), _stream_ptr(stream)),
                    "form_residual_noalloc")

    def form_residual_timed(self, u, res, stream=None):
        """(ms face kernel, ms volume kernel) from CUDA events; synchronises"""
        a, b = C.c_double(), C.c_double()
        self._check(lib().icx_form_residual_timed(self._h, _ptr(u), _ptr(res), _stream_ptr(stream), C.byref(a),
                                                  C.byref(b)), "form_residual_timed")
        return a.value, b.value

    def jacobian_pattern(self):
        E = self.layout.n_elem
        rowptr = np.zeros(E + 1, dtype=np.int32)
        colidx = np.zeros(self.layout.nnz_blocks, dtype=np.int32)
        self._check(lib().icx_jacobian_pattern(self._h, _ptr(rowptr), _ptr(colidx)), "jacobian_pattern")
        return rowptr, colidx

    def form_jacobian_fd(self, u, res, vals, eps=0.0, stream=None):
        self._check(lib().icx_form_jacobian_fd(self._h, _ptr(u), _ptr(res), _ptr(vals), eps, _stream_ptr(stream)),
                    "form_jacobian_fd")

    def form_jacobian_fd_f32(self, u, res, vals32, stream=None):
        """the FD Jacobian with FP32 flux quadrature into FP32 BSR values
        (res = R(u) in FP64)"""
        self._check(lib().icx_form_jacobian_fd_f32(self._h, _ptr(u), _ptr(res), _ptr(vals32), _stream_ptr(stream)),
                    "form_jacobian_fd_f32")

    def bsr_spmv(self, vals, x, y, stream=None):
        self._check(lib().icx_bsr_spmv(self._h, _ptr(vals), _ptr(x), _ptr(y), _stream_ptr(stream)), "bsr_spmv")

    def gmres_solve(self, vals, b, x, restart=30, maxit=2000, rtol=1e-5, preconditioner=2, stream=None):
        """(iterations, relative residual, converged) of J x = b"""
        it, rr = C.c_int(), C.c_double()
        st = lib().icx_gmres_solve(self._h, _ptr(vals), _ptr(b), _ptr(x), restart, maxit, rtol, preconditioner,
                                   C.byref(it), C.byref(rr), _stream_ptr(stream))
        if st not in (0, 5):
            self._check(st, "gmres_solve")
        return it.value, rr.value, st == 0

    # --- MDG-ICE -----------------------------------------------------------
    def mdg_select(self, traces, hyper_rectangle=True):
        tr = np.ascontiguousarray(traces, dtype=np.int32)
        self._check(lib().icx_mdg_select(self._h, len(tr), _ptr(tr), int(hyper_rectangle)), "mdg_select")
        ns, ng = C.c_int(), C.c_int()
        self._check(lib().icx_mdg_info(self._h, C.byref(ns), C.byref(ng)), "mdg_info")
        self.mdg_nsel, self.mdg_ngeo = ns.value, ng.value
        return ns.value, ng.value

    def mdg_selected_nodes(self):
        out = np.zeros(self.mdg_nsel, dtype=np.int32)
        self._check(lib().icx_mdg_selected_nodes(self._h, _ptr(out)), "mdg_selected_nodes")
        return out

    def mdg_get_x(self):
        x = np.zeros(self.mdg_ngeo)
        self._check(lib().icx_mdg_get_x(self._h, _ptr(x)), "mdg_get_x")
        return x

    def mdg_set_x(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        self._check(lib().icx_mdg_set_x(self._h, _ptr(x)), "mdg_set_x")

    def form_residual_mdg(self, u, x, res, ic, stream=None):
        xp = None if x is None else _ptr(np.ascontiguousarray(x, dtype=np.float64))
        self._check(lib().icx_form_residual_mdg(self._h, _ptr(u), xp, _ptr(res), _ptr(ic), _stream_ptr(stream)),
                    "form_residual_mdg")

    def mdg_jacobian_pattern(self):
        nr, nc, nz = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._check(lib().icx_mdg_jacobian_pattern(self._h, C.byref(nr), C.byref(nc), C.byref(nz), None, None),
                    "mdg_jacobian_pattern")
        rowptr = np.zeros(nr.value + 1, dtype=np.int32)
        colidx = np.zeros(nz.value, dtype=np.int32)
        self._check(lib().icx_mdg_jacobian_pattern(self._h, C.byref(nr), C.byref(nc), C.byref(nz), _ptr(rowptr),
                                                   _ptr(colidx)), "mdg_jacobian_pattern")
        return nr.value, nc.value, rowptr, colidx

    def form_jacobian_mdg_fd(self, u, res, ic, vals, eps=0.0, stream=None):
        self._check(lib().icx_form_jacobian_mdg_fd(self._h, _ptr(u), _ptr(res), _ptr(ic), _ptr(vals), eps,
                                                   _stream_ptr(stream)), "form_jacobian_mdg_fd")

    def explicit_solve(self, u, options=None):
        """advance u (device, FP64) in place with an explicit time stepper
        (ExplicitEuler / RK3TVD / RK3SSP); returns the ExplicitReport"""
        opt = options or default_explicit_options()
        rep = ExplicitReport()
        self._check(lib().icx_explicit_solve(self._h, _ptr(u), C.byref(opt), C.byref(rep)), "explicit_solve")
        return rep

    def mass_inverse_apply(self, r, out, stream=None):
        """out = M^-1 r element by element (device arrays)"""
        self._check(lib().icx_mass_inverse_apply(self._h, _ptr(r), _ptr(out), _stream_ptr(stream)),
                    "mass_inverse_apply")

    def write_restart(self, u, k, rank=0, directory=None):
        """write_restart: <directory>/restart<k>_<rank> (directory None:
        RESTART under the working directory) from u (device, FP64)"""
        d = None if directory is None else str(directory).encode()
        self._check(lib().icx_write_restart(self._h, _ptr(u), int(k), int(rank), d), "write_restart")

    def read_restart(self, u, name, rank=0, directory=None):
        """read_restart: moves the mesh nodes to the file's coordinates and
        fills u (device, FP64) from <directory>/<name>_<rank>"""
        d = None if directory is None else str(directory).encode()
        self._check(lib().icx_read_restart(self._h, _ptr(u), name.encode(), int(rank), d), "read_restart")

    @staticmethod
    def _names(names):
        if names is None:
            return None
        arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
        return arr

    def write_vtu(self, u, itime, kind=0, directory=None, collection=None, names=None, precision=8):
        """PVDWriter::write_vtu of u (kind VTU_SOLUTION) or of its residual
        and the residual's domain and trace parts (kind VTU_RESIDUAL)"""
        d = None if directory is None else str(directory).encode()
        cn = None if collection is None else collection.encode()
        self._check(lib().icx_write_vtu(self._h, _ptr(u), int(kind), int(itime), d, cn, self._names(names),
                                        int(precision)), "write_vtu")

    def write_vtu_mdg(self, ic, itime, directory=None, collection=None, names=None, precision=8):
        """the MDG interface-conservation residual ic (device, [selected node][neq])
        as an isoparametric nodal field"""
        d = None if directory is None else str(directory).encode()
        cn = None if collection is None else collection.encode()
        self._check(lib().icx_write_vtu_mdg(self._h, _ptr(ic), int(itime), d, cn, self._names(names),
                                            int(precision)), "write_vtu_mdg")

    def krylov_samples(self, vals, b, x, samples, every=8, restart=30, maxit=2000, rtol=1e-5, preconditioner=2):
        """GMRES on J = vals from a zero guess that copies restart residuals and
        every `every`-th Arnoldi vector into samples ([cap][n_dof] FP64 device
        tensor); returns (n_samples, iterations, relres)"""
        ns, it, rr = C.c_int(), C.c_int(), C.c_double()
        st = lib().icx_krylov_samples(self._h, _ptr(vals), _ptr(b), _ptr(x), restart, maxit, rtol, preconditioner,
                                      every, samples.shape[0], _ptr(samples), C.byref(ns), C.byref(it), C.byref(rr))
        self._check(st, "krylov_samples")
        return ns.value, it.value, rr.value

    def lpc_attach(self, model):
        """use a LearnedPreconditioner for Newton preconditioner 5 (None: detach)"""
        self._check(lib().icx_lpc_attach(self._h, None if model is None else model._h), "lpc_attach")
        self._lpc = model

    def lpc_forward(self, vals, corr=None):
        """the attached model's correction blocks for Jacobian vals"""
        self._check(lib().icx_lpc_forward(self._h, _ptr(vals), None if corr is None else _ptr(corr)), "lpc_forward")

    def lpc_train(self, vals, samples, n_samples, steps=100, batch=4, random=0, sweeps=1, lr=1e-3, seed=0):
        """Adam steps of the attached model on Jacobian vals and residual
        samples (`random` of each batch's vectors are seeded Gaussian ones)"""
        o = LpcTrainOptions(steps, batch, random, sweeps, lr, seed)
        rep = LpcTrainReport()
        self._check(lib().icx_lpc_train(self._h, _ptr(vals), int(n_samples), _ptr(samples), C.byref(o),
                                        C.byref(rep)), "lpc_train")
        return rep

    def lpc_calibrate(self, vals, samples, n_samples, sweeps=0):
        """(sum <a,b>/|r|^2, sum |b|^2/|r|^2, sum |a|^2/|r|^2) over the samples
        r, with a = r - J y, b = J C y, y the base preconditioner's output"""
        out = (C.c_double * 3)()
        self._check(lib().icx_lpc_calibrate(self._h, _ptr(vals), int(n_samples), _ptr(samples), int(sweeps), out),
                    "lpc_calibrate")
        return tuple(out)

    def mfnk_solve(self, u, options=None):
        """matrix-free Newton-Krylov on u (device, FP64, in place); returns the report"""
        opt = options or default_newton_options()
        rep = NewtonReport()
        st = lib().icx_mfnk_solve(self._h, _ptr(u), C.byref(opt), C.byref(rep))
        if st not in (0, 5):
            self._check(st, "mfnk_solve")
        return rep

    def newton_solve(self, u, options=None):
        opt = options or default_newton_options()
        rep = NewtonReport()
        st = lib().icx_newton_solve(self._h, _ptr(u), C.byref(opt), C.byref(rep))
        if st not in (0, 5):
            self._check(st, "newton_solve")
        return rep


VTU_SOLUTION = 0
VTU_RESIDUAL = 1


class LearnedPreconditioner:
    """icx_lpc: the MLP of the learned block preconditioner (block size bs,
    `hidden` units per hidden layer) on one device."""

    def __init__(self, bs, hidden=256, device=0, seed=0):
        self._h = C.c_void_p()
        st = lib().icx_lpc_create(C.byref(self._h), device, bs, hidden, seed)
        if st != 0:
            raise IcxError(st, "icx_lpc_create")
        self.bs, self.hidden, self.device = bs, hidden, device
        self.sweeps = None
        self.ilu_tile = None

    def close(self):
        if self._h:
            lib().icx_lpc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_params(self):
        n = C.c_longlong()
        lib().icx_lpc_info(self._h, None, None, C.byref(n), None)
        return n.value

    @property
    def steps(self):
        n = C.c_longlong()
        lib().icx_lpc_info(self._h, None, None, None, C.byref(n))
        return n.value

    def get_params(self):
        p = np.zeros(self.n_params, dtype=np.float32)
        st = lib().icx_lpc_get_params(self._h, p.ctypes.data_as(C.c_void_p))
        if st != 0:
            raise IcxError(st, "icx_lpc_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"{p.size} parameters, the model has {self.n_params}")
        st = lib().icx_lpc_set_params(self._h, p.ctypes.data_as(C.c_void_p))
        if st != 0:
            raise IcxError(st, "icx_lpc_set_params")

    def save(self, path, sweeps=None, ilu_tile=None):
        """parameters and shape (and the base preconditioner the model was
        trained on: Jacobi sweeps, i.e. the pc_sweeps to run it with, and the
        ILU tile side) as a compressed .npz"""
        extra = {} if sweeps is None else {"sweeps": sweeps}
        if ilu_tile is not None:
            extra["ilu_tile"] = ilu_tile
        np.savez_compressed(path, bs=self.bs, hidden=self.hidden, params=self.get_params(), **extra)

    @classmethod
    def load(cls, path, device=0):
        z = np.load(path)
        m = cls(int(z["bs"]), int(z["hidden"]), device)
        m.set_params(z["params"])
        m.sweeps = int(z["sweeps"]) if "sweeps" in z.files else None
        m.ilu_tile = int(z["ilu_tile"]) if "ilu_tile" in z.files else None
        return m


def batch(parts, device=0):
    """one Context holding the set-up Contexts `parts` side by side (the batch
    keeps them alive); `elem_offsets` gives each part's first element, then the
    total"""
    b = Context.__new__(Context)
    b._h = C.c_void_p()
    b._keep = list(parts)
    arr = (C.c_void_p * len(parts))(*[p._h.value for p in parts])
    st = lib().icx_batch_create(C.byref(b._h), device, len(parts), arr)
    if st != 0:
        raise IcxError(st, "batch_create")
    off = (C.c_int * (len(parts) + 1))()
    b._check(lib().icx_batch_offsets(b._h, off), "batch_offsets")
    b.elem_offsets = list(off)
    lay = LayoutInfo()
    b._check(lib().icx_get_layout(b._h, C.byref(lay)), "get_layout")
    b.layout = lay
    return b


class ProblemSet:
    """icx_pset: independent problems of uneven mesh size and basis order
    (set-up Contexts, kept alive by the set), each solved by its own Newton
    iteration with every kernel launched once per basis order for all parts.
    `offsets[k]` is part k's first unknown in the set's vectors (the parts
    are stored by basis order), `lengths[k]` its unknowns, `offsets[-1]` the
    total."""

    def __init__(self, parts, device=0):
        self._h = C.c_void_p()
        self._keep = list(parts)
        arr = (C.c_void_p * len(parts))(*[p._h.value for p in parts])
        st = lib().icx_pset_create(C.byref(self._h), device, len(parts), arr)
        if st != 0:
            raise IcxError(st, "pset_create")
        off = (C.c_longlong * (len(parts) + 1))()
        self._check(lib().icx_pset_offsets(self._h, off), "pset_offsets")
        self.offsets = list(off)
        self.lengths = [p.layout.n_dof for p in parts]
        self.n_parts = len(parts)

    def _check(self, st, what):
        if st != 0:
            raise IcxError(st, f"{what}: {lib().icx_pset_last_error(self._h).decode()}")

    def close(self):
        if self._h:
            lib().icx_pset_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def gather(self, vectors):
        """one host vector in the set's layout from the parts' vectors"""
        out = np.zeros(self.offsets[-1])
        for k, v in enumerate(vectors):
            out[self.offsets[k]:self.offsets[k] + self.lengths[k]] = v
        return out

    def part(self, x, k):
        return x[self.offsets[k]:self.offsets[k] + self.lengths[k]]

    def residual(self, u, res):
        self._check(lib().icx_pset_residual(self._h, _ptr(u), _ptr(res)), "pset_residual")

    def newton_solve(self, u, options=None):
        """(reports per part, PsetStats); a part that does not converge shows
        in its report (the call itself raises only on other errors)"""
        opt = options or default_newton_options()
        reps = (NewtonReport * self.n_parts)()
        stats = PsetStats()
        st = lib().icx_pset_newton_solve(self._h, _ptr(u), C.byref(opt), reps, C.byref(stats))
        if st not in (0, 5):
            self._check(st, "pset_newton_solve")
        return list(reps), stats


def default_explicit_options(**kw):
    opt = ExplicitOptions()
    st = lib().icx_explicit_default_options(C.byref(opt))
    if st != 0:
        raise IcxError(st, "explicit_default_options")
    for k, v in kw.items():
        setattr(opt, k, v)
    return opt


def gemm_bf16_nt(A, B, bias=None, relu=False, out32=None, out16=None, accumulate=False, splits=1):
    """out = A . B^T (+ bias, ReLU) on the tensor cores; A [M, K] and B [N, K]
    BF16 CUDA tensors, out32 FP32 and/or out16 BF16 [M, N] (accumulate: out32 +=)"""
    M, K = A.shape
    N = B.shape[0]
    st = lib().icx_gemm_bf16_nt(M, N, K, _ptr(A), A.stride(0), _ptr(B), B.stride(0),
                                _ptr(bias) if bias is not None else None, int(relu),
                                _ptr(out32) if out32 is not None else None, out32.stride(0) if out32 is not None else 0,
                                _ptr(out16) if out16 is not None else None, out16.stride(0) if out16 is not None else 0,
                                int(accumulate), int(splits), None)
    if st != 0:
        raise IcxError(st, "gemm_bf16_nt")


def workload_fn(name):
    """address of an exported workload callback (icx_wl_*) as an icx_point_fn"""
    return C.cast(getattr(lib(), "icx_wl_" + name), POINT_FN)


def default_newton_options():
    opt = NewtonOptions()
    st = lib().icx_newton_default_options(C.byref(opt))
    if st != 0:
        raise IcxError(st, "newton_default_options")
    return opt


class LMOptions(C.Structure):
    _fields_ = [("tau_abs", C.c_double), ("tau_rel", C.c_double), ("kmax", C.c_int), ("lambda_u", C.c_double),
                ("lambda_b", C.c_double), ("linesearch", C.c_int), ("ls_max_it", C.c_int),
                ("ls_alpha_initial", C.c_double), ("ls_alpha_max", C.c_double), ("ls_alpha_min", C.c_double),
                ("gmres_restart", C.c_int), ("gmres_max_it", C.c_int), ("gmres_rtol", C.c_double),
                ("max_rejections", C.c_int), ("verbosity", C.c_int), ("explicit_subproblem", C.c_int),
                ("lambda_lag", C.c_double), ("step_only", C.c_int)]


class LMReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rejections", C.c_int), ("r0", C.c_double),
                ("r_final", C.c_double), ("linear_iterations_total", C.c_int),
                ("residual_history", C.c_double * 64), ("alpha_history", C.c_double * 64),
                ("linear_relres_max", C.c_double)]


def default_lm_options():
    o = LMOptions()
    L = lib()
    L.icx_lm_default_options.restype = C.c_int
    L.icx_lm_default_options.argtypes = [C.POINTER(LMOptions)]
    st = L.icx_lm_default_options(C.byref(o))
    if st != 0:
        raise IcxError(st, "lm_default_options")
    return o


def lm_solve(ctx, u, x, options=None):
    """CorriganLM::solve: u (device tensor) and x (numpy, host) updated in place"""
    L = lib()
    L.icx_lm_solve.restype = C.c_int
    L.icx_lm_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LMOptions), C.POINTER(LMReport)]
    opt = options or default_lm_options()
    rep = LMReport()
    assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"]
    st = L.icx_lm_solve(ctx._h, _ptr(u), _ptr(x), C.byref(opt), C.byref(rep))
    if st not in (0, 5):
        ctx._check(st, "lm_solve")
    return rep
