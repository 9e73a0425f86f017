"""ctypes bindings of the CPU oracle (oracle/liboracle.so) and of the
reference CPU build (oracle/_ref/libiceicle_ref.so), plus the seeded problem
builders the parity tests use. Test infrastructure only."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libiceicle_ref.so")

POINT_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p)

BC_NEUMANN, BC_DIRICHLET, BC_EXTRAPOLATION = 2, 3, 4


class Problem(C.Structure):
    """Same layout as orc_problem (oracle/oracle.h) and ref_problem."""
    _fields_ = [
        ("pde", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("geo_order", C.c_int), ("p", C.c_int),
        ("xmin", C.c_double * 2), ("xmax", C.c_double * 2), ("bctype", C.c_int * 4), ("bcflag", C.c_int * 4),
        ("interior_penalty", C.c_int), ("sigma_ic", C.c_double), ("mu", C.c_double),
        ("a", C.c_double * 2), ("b", C.c_double * 2), ("gamma", C.c_double), ("Pr", C.c_double),
        ("ns_mu", C.c_double),
        ("n_dirichlet", C.c_int), ("dirichlet", POINT_FN * 8), ("dirichlet_user", C.c_void_p * 8),
        ("n_neumann", C.c_int), ("neumann", POINT_FN * 8), ("neumann_user", C.c_void_p * 8),
        ("source", POINT_FN), ("source_user", C.c_void_p), ("spacetime", C.c_int), ("basis", C.c_int),
        ("ns_flux", C.c_int), ("n_wall", C.c_int), ("wall_T", C.c_double * 8),
        ("fs_rho", C.c_double), ("fs_u_inf", C.c_double), ("fs_dir", C.c_double * 2), ("fs_T", C.c_double),
        ("ns_visc", C.c_int), ("suth", C.c_double * 3),
    ]


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class _Lib:
    def __init__(self, path, prefix):
        self.lib = C.CDLL(path)
        self.prefix = prefix

    def fn(self, name):
        return getattr(self.lib, self.prefix + name)


_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        _oracle = _Lib(ORACLE_SO, "orc_")
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = _Lib(REF_SO, "ref_")
    return _ref


def neq(pb):
    return 1 if pb.pde == 0 else 4


def sizes(pb):
    nb = (pb.p + 1) ** 2
    E = pb.nx * pb.ny
    return E, nb, E * nb * neq(pb)


def lattice_coords(pb):
    """Equispaced geometry-node lattice, x fastest (n_nodes x 2)."""
    g = pb.geo_order
    nnx, nny = pb.nx * g + 1, pb.ny * g + 1
    ix, iy = np.meshgrid(np.arange(nnx), np.arange(nny))
    x = pb.xmin[0] + (pb.xmax[0] - pb.xmin[0]) * ix.ravel() / (pb.nx * g)
    y = pb.xmin[1] + (pb.xmax[1] - pb.xmin[1]) * iy.ravel() / (pb.ny * g)
    return np.ascontiguousarray(np.stack([x, y], axis=1))


def perturb_smooth(pb, coord, amp_frac, seed):
    """Seeded smooth displacement of every node that keeps the domain boundary:
    d = A h sin(pi xs) sin(pi ys) (c1 sin(2 pi k.xs + ph)), xs in [0,1]^2."""
    rng = np.random.default_rng(seed)
    hx = (pb.xmax[0] - pb.xmin[0]) / pb.nx
    hy = (pb.xmax[1] - pb.xmin[1]) / pb.ny
    xs = (coord[:, 0] - pb.xmin[0]) / (pb.xmax[0] - pb.xmin[0])
    ys = (coord[:, 1] - pb.xmin[1]) / (pb.xmax[1] - pb.xmin[1])
    bump = np.sin(np.pi * xs) * np.sin(np.pi * ys)
    k = rng.integers(1, 4, size=(2, 2))
    ph = rng.uniform(0, 2 * np.pi, size=2)
    out = coord.copy()
    out[:, 0] += amp_frac * hx * bump * np.sin(2 * np.pi * (k[0, 0] * xs + k[0, 1] * ys) + ph[0])
    out[:, 1] += amp_frac * hy * bump * np.sin(2 * np.pi * (k[1, 0] * xs + k[1, 1] * ys) + ph[1])
    return np.ascontiguousarray(out)


def basis_node_coords(pb, coord):
    """physical coordinates of the Lagrange basis nodes [E][nb][2] (oracle)"""
    E, nb, N = sizes(pb)
    xy = np.zeros((E, nb, 2))
    rc = oracle().fn("basis_node_coords")(C.byref(pb), _ptr(np.ascontiguousarray(coord)), _ptr(xy))
    assert rc == 0, rc
    return xy


def residual(lib, pb, coord, u):
    E, nb, N = sizes(pb)
    r = np.zeros(N)
    rc = lib.fn("form_residual")(C.byref(pb), _ptr(coord), _ptr(np.ascontiguousarray(u, dtype=np.float64)), _ptr(r))
    assert rc == 0, rc
    return r


def topology(lib, pb):
    E = pb.nx * pb.ny
    ng = (pb.geo_order + 1) ** 2
    nf = (pb.nx - 1) * pb.ny + pb.nx * (pb.ny - 1) + 2 * pb.nx + 2 * pb.ny
    conn = np.zeros(E * ng, dtype=np.int32)
    faces = np.zeros(nf * 7, dtype=np.int32)
    nint = C.c_int()
    got = lib.fn("mesh_topology")(C.byref(pb), _ptr(conn), _ptr(faces), C.byref(nint))
    return conn.reshape(E, ng), faces[: got * 7].reshape(got, 7), nint.value


def bsr_pattern(pb):
    E = pb.nx * pb.ny
    rowptr = np.zeros(E + 1, dtype=np.int32)
    colidx = np.zeros(5 * E, dtype=np.int32)
    nnz = oracle().fn("bsr_pattern")(C.byref(pb), _ptr(rowptr), _ptr(colidx))
    return rowptr, colidx[:nnz].copy()


def jacobian_bsr(pb, coord, u):
    E, nb, N = sizes(pb)
    bs = nb * neq(pb)
    rowptr, colidx = bsr_pattern(pb)
    vals = np.zeros(len(colidx) * bs * bs)
    r = np.zeros(N)
    rc = oracle().fn("form_jacobian_fd")(C.byref(pb), _ptr(coord), _ptr(np.ascontiguousarray(u)), _ptr(r),
                                         _ptr(rowptr), _ptr(colidx), _ptr(vals))
    assert rc == 0, rc
    return r, rowptr, colidx, vals.reshape(-1, bs, bs)


def ref_jacobian_dense(pb, coord, u):
    E, nb, N = sizes(pb)
    r = np.zeros(N)
    J = np.zeros((N, N))
    rc = ref().fn("form_jacobian_dense")(C.byref(pb), _ptr(coord), _ptr(np.ascontiguousarray(u)), _ptr(r), _ptr(J))
    assert rc == 0, rc
    return r, J


def bsr_to_dense(rowptr, colidx, vals):
    E = len(rowptr) - 1
    bs = vals.shape[1]
    J = np.zeros((E * bs, E * bs))
    for r in range(E):
        for k in range(rowptr[r], rowptr[r + 1]):
            c = colidx[k]
            J[r * bs:(r + 1) * bs, c * bs:(c + 1) * bs] = vals[k]
    return J


# ------------------------------------------------------------------ MDG-ICE
def mdg_select(lib, pb, coord, traces, hyper=True):
    nn = (pb.nx * pb.geo_order + 1) * (pb.ny * pb.geo_order + 1)
    tr = np.ascontiguousarray(traces, dtype=np.int32)
    sel = np.zeros(nn, dtype=np.int32)
    x = np.zeros(2 * nn)
    nsel = C.c_int()
    ngeo = lib.fn("mdg_select")(C.byref(pb), _ptr(coord), len(tr), _ptr(tr), int(hyper), C.byref(nsel), _ptr(sel),
                                _ptr(x))
    return sel[: nsel.value].copy(), x[:ngeo].copy()


def mdg_residual(lib, pb, coord, traces, u, x, hyper=True):
    E, nb, N = sizes(pb)
    sel, _ = mdg_select(lib, pb, coord, traces, hyper)
    tr = np.ascontiguousarray(traces, dtype=np.int32)
    ux = np.ascontiguousarray(np.concatenate([u, x]))
    out = np.zeros(N + len(sel) * neq(pb))
    if lib.prefix == "ref_":
        rc = lib.fn("mdg_residual")(C.byref(pb), _ptr(coord), len(tr), _ptr(tr), int(hyper), _ptr(ux), len(ux),
                                    _ptr(out), len(out))
    else:
        rc = lib.fn("mdg_residual")(C.byref(pb), _ptr(coord), len(tr), _ptr(tr), int(hyper), _ptr(ux), _ptr(out))
    assert rc == 0, rc
    return out


def mdg_jacobian_dense(lib, pb, coord, traces, u, x, hyper=True):
    E, nb, N = sizes(pb)
    sel, _ = mdg_select(lib, pb, coord, traces, hyper)
    tr = np.ascontiguousarray(traces, dtype=np.int32)
    nres = N + len(sel) * neq(pb)
    out = np.zeros(nres)
    J = np.zeros((nres, N + len(x)))
    u = np.ascontiguousarray(u)
    x = np.ascontiguousarray(x)
    if lib.prefix == "ref_":
        rc = lib.fn("mdg_jacobian_dense")(C.byref(pb), _ptr(coord), len(tr), _ptr(tr), int(hyper), _ptr(u), _ptr(x),
                                          len(x), _ptr(out), nres, _ptr(J))
    else:
        rc = lib.fn("mdg_jacobian_dense")(C.byref(pb), _ptr(coord), len(tr), _ptr(tr), int(hyper), _ptr(u), _ptr(x),
                                          _ptr(out), _ptr(J))
    assert rc == 0, rc
    return out, J


def mass_matrices(lib, pb, coord):
    """element mass matrices [E][nb][nb] (oracle or reference build)"""
    E, nb, N = sizes(pb)
    M = np.zeros((E, nb, nb))
    rc = lib.fn("mass_matrices")(C.byref(pb), _ptr(coord), _ptr(M))
    assert rc == 0, rc
    return M


def explicit_solve(lib, pb, coord, u, scheme, dt_kind=0, dt=0.0, cfl=0.3, term_kind=0, ntime=1, tfinal=0.0):
    """run an explicit solver (0 Euler, 1 TVD-RK3, 2 SSP-RK3) from u; returns
    (u, steps, time)"""
    uu = np.ascontiguousarray(u, dtype=np.float64).copy()
    steps, t = C.c_int(), C.c_double()
    rc = lib.fn("explicit_solve")(C.byref(pb), _ptr(coord), _ptr(uu), int(scheme), int(dt_kind), C.c_double(dt),
                                  C.c_double(cfl), int(term_kind), int(ntime), C.c_double(tfinal), C.byref(steps),
                                  C.byref(t))
    assert rc == 0, rc
    return uu, steps.value, t.value


def ref_write_restart(pb, coord, u, k, directory):
    """the reference's write_restart run in `directory` (writes
    directory/RESTART/restart<k>_0)"""
    uu = np.ascontiguousarray(u, dtype=np.float64)
    rc = ref().fn("write_restart")(C.byref(pb), _ptr(coord), _ptr(uu), int(k), str(directory).encode())
    assert rc == 0, rc


def ref_read_restart(pb, name, directory):
    """the reference's read_restart run in `directory`: (coords, u)"""
    E, nb, N = sizes(pb)
    nn = (pb.nx * pb.geo_order + 1) * (pb.ny * pb.geo_order + 1)
    coord = np.zeros(2 * nn)
    u = np.zeros(N)
    rc = ref().fn("read_restart")(C.byref(pb), name.encode(), str(directory).encode(), _ptr(coord), _ptr(u))
    assert rc == 0, rc
    return coord, u


def ref_write_vtu(pb, coord, u, kind, itime, directory, collection):
    """PVDWriter::write_vtu of the reference: kind 0 fields of u, 1 residuals"""
    uu = np.ascontiguousarray(u, dtype=np.float64)
    rc = ref().fn("write_vtu")(C.byref(pb), _ptr(coord), _ptr(uu), int(kind), int(itime), str(directory).encode(),
                               collection.encode())
    assert rc == 0, rc


def ref_write_vtu_mdg(pb, coord, traces, hyper, ic, itime, directory, collection):
    """the reference driver's MDG residual VTU (ic: [selected node][neq])"""
    tr = np.ascontiguousarray(traces, dtype=np.int32)
    icc = np.ascontiguousarray(ic, dtype=np.float64)
    rc = ref().fn("write_vtu_mdg")(C.byref(pb), _ptr(coord), len(tr), _ptr(tr), int(hyper), _ptr(icc), int(itime),
                                   str(directory).encode(), collection.encode())
    assert rc == 0, rc
