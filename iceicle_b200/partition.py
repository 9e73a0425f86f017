"""Element-row partitioning of a uniform nx x ny quad mesh over ranks, and the
halo exchange before each residual.

Reference: partition_mesh (src/FiniteElement/include/iceicle/mesh/
mesh_partition.hpp:26-44: the identity on one rank, METIS k-way on the
element dual graph otherwise) and the halo exchange inside form_residual
(src/solvers/include/iceicle/form_residual.hpp:87-135: for each element
owned by another rank that shares a face with this rank, MPI_Send /
MPI_Recv of its nb * neq coefficients, rank by rank).

Here rank r owns the element rows [j0, j1), a contiguous block of the
global element numbering iel = i + nx j. It also holds a copy of the row
below and the row above that block wherever another rank owns them (ghost
rows). Its context is the sub-mesh of rows [g0, g1), built on the global
geometry nodes of those rows. Every face of an owned element, partition
faces included, is then a face of the sub-mesh with the same geometry and
the same neighbour data as in the global mesh, so the owned entries of the
sub-mesh residual are the global residual's entries. Only a ghost row's own
entries differ, because its outer side is an artificial boundary; they are
not used.

The exchange sends one owned boundary row to each neighbouring rank per
residual: nx * nb * neq values, contiguous in the DOF layout
u[(iel * nb + idof) * neq + ieq]. It runs over torch.distributed
point-to-point operations (NCCL between GPUs, gloo on the CPU).
"""


def strip_rows(ny, nranks, rank):
    """owned element rows [j0, j1) of `rank`: contiguous, balanced to one row"""
    if nranks < 1 or not 0 <= rank < nranks:
        raise ValueError("rank out of range")
    if ny < nranks:
        raise ValueError(f"{ny} element rows cannot be split over {nranks} ranks")
    q, rem = divmod(ny, nranks)
    j0 = rank * q + min(rank, rem)
    return j0, j0 + q + (1 if rank < rem else 0)


class StripPlan:
    """the rows, elements, nodes and DOFs a rank owns and holds"""

    def __init__(self, nx, ny, nranks, rank, geo_order):
        self.nx, self.ny, self.nranks, self.rank, self.g = nx, ny, nranks, rank, geo_order
        self.j0, self.j1 = strip_rows(ny, nranks, rank)
        self.g0 = self.j0 - 1 if rank > 0 else 0
        self.g1 = self.j1 + 1 if rank < nranks - 1 else ny
        self.below = rank - 1 if rank > 0 else None  # neighbour owning row j0 - 1
        self.above = rank + 1 if rank < nranks - 1 else None  # neighbour owning row j1

    @property
    def rows(self):
        """element rows of the sub-mesh (owned + ghosts)"""
        return self.g1 - self.g0

    def owned_elements(self):
        """owned elements in the sub-mesh numbering, [e0, e1)"""
        return (self.j0 - self.g0) * self.nx, (self.j1 - self.g0) * self.nx

    def node_range(self):
        """global geometry-node indices [n0, n1) of the sub-mesh (x fastest,
        (nx g + 1) nodes per node row; node rows g0 g .. g1 g)"""
        w = self.nx * self.g + 1
        return self.g0 * self.g * w, (self.g1 * self.g + 1) * w

    def global_dofs(self, bs):
        """global DOF range [d0, d1) of the sub-mesh's elements, bs = nb * neq"""
        return self.g0 * self.nx * bs, self.g1 * self.nx * bs

    def owned_dofs(self, bs):
        """owned DOFs in the sub-mesh vector, [d0, d1)"""
        e0, e1 = self.owned_elements()
        return e0 * bs, e1 * bs

    def halo(self, bs):
        """(peer, send range, receive range) per neighbour, ranges in the
        sub-mesh vector: the owned boundary row goes out, the peer's row
        lands in the ghost row"""
        row = self.nx * bs
        lo = self.j0 - self.g0  # local index of the first owned row
        hi = self.j1 - self.g0  # local index of the ghost row above, if any
        out = []
        if self.below is not None:
            out.append((self.below, (lo * row, (lo + 1) * row), (0, row)))
        if self.above is not None:
            out.append((self.above, ((hi - 1) * row, hi * row), (hi * row, (hi + 1) * row)))
        return out


def halo_exchange(plan, u_local, bs, group=None):
    """fills the ghost rows of u_local (1-D tensor of the sub-mesh DOFs) with
    the neighbours' owned boundary rows; every rank of a partition calls it
    together. Returns the number of values received."""
    import torch.distributed as dist
    ops = []
    n = 0
    for peer, (s0, s1), (r0, r1) in plan.halo(bs):
        ops.append(dist.P2POp(dist.isend, u_local[s0:s1], peer, group))
        ops.append(dist.P2POp(dist.irecv, u_local[r0:r1], peer, group))
        n += r1 - r0
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return n


def sub_coords(plan, global_coords):
    """the sub-mesh's geometry nodes, sliced from the global node array [n, 2]"""
    n0, n1 = plan.node_range()
    return global_coords[n0:n1].copy()


class StripResidual:
    """form_residual on a partitioned mesh: the halo exchange, then the
    residual of the rank's sub-mesh context (its owned entries are the
    global residual's)"""

    def __init__(self, ctx, plan, group=None):
        self.ctx, self.plan, self.group = ctx, plan, group
        L = ctx.layout
        self.bs = L.block_size
        if L.n_elem != plan.rows * plan.nx:
            raise ValueError("context does not match the partition's sub-mesh")

    def owned(self, v):
        d0, d1 = self.plan.owned_dofs(self.bs)
        return v[d0:d1]

    def __call__(self, u_local, res_local, stream=None):
        """exchange, then the residual on `stream` (torch's current stream when
        None). The exchange is issued on that stream too, so its receives are
        ordered before the residual kernels whatever stream the caller uses."""
        import torch
        if stream is None or not u_local.is_cuda:
            halo_exchange(self.plan, u_local, self.bs, self.group)
            self.ctx.form_residual(u_local, res_local, stream)
            return
        with torch.cuda.stream(stream):
            halo_exchange(self.plan, u_local, self.bs, self.group)
            self.ctx.form_residual(u_local, res_local, stream)


class StripKrylov:
    """J du = r on element-row strips: the linear solve of the Newton step of
    a partitioned mesh (the reference's PETSc KSP over MPI ranks,
    petsc_newton.hpp:159-183). Vectors are a rank's owned DOFs; the rank's
    block rows of J are those of its sub-mesh context (owned rows and the
    columns of the ghost rows).

    * product y = J x: the halo exchange of x's boundary rows into the ghost
      rows (one message per neighbour, as before a residual), the local
      block-row product, the owned rows of the result;
    * inner products: the rank's partial sums, then one all-reduce of all the
      Gram-Schmidt coefficients of a step (one collective per pass, not one
      per vector);
    * preconditioner: block-Jacobi across ranks, ILU(0) of each rank's owned
      block (couplings to ghost rows dropped), PETSc's parallel default
      (bjacobi with ilu sub-solves).

    `local_mv(x_ext, y_ext)` multiplies by the rank's block rows on the
    sub-mesh vector; `local_pc(x_own, y_own)` applies the rank's owned-block
    preconditioner. On GPUs these are the context's BSR product and
    icx_pc_apply with the owned elements grouped (StripKrylov.for_context);
    the CPU tests pass restatements. Restarted GMRES(m), right-preconditioned,
    classical Gram-Schmidt with one re-orthogonalisation, Hessenberg and
    Givens on the host in FP64: the single-GPU solver's algorithm, so one rank
    reproduces it."""

    def __init__(self, plan, bs, local_mv, local_pc=None, group=None):
        self.plan, self.bs, self.group = plan, bs, group
        self.local_mv, self.local_pc = local_mv, local_pc
        self.d0, self.d1 = plan.owned_dofs(bs)
        self.n_ext = plan.rows * plan.nx * bs

    @classmethod
    def for_context(cls, ctx, plan, vals, precision=0, group=None):
        """the GPU form over a strip context: BSR product with the Jacobian
        values `vals`, block-ILU(0) of the owned elements (every ghost row in
        a group of its own)"""
        import numpy as np
        L = ctx.layout
        e0, e1 = plan.owned_elements()
        groups = np.arange(L.n_elem, dtype=np.int32) + 1
        groups[e0:e1] = 0
        ctx.set_ilu_groups(groups)
        ctx.pc_factor(vals, precision)
        bs = L.block_size
        d0, d1 = plan.owned_dofs(bs)
        import torch
        buf_in = torch.zeros(L.n_dof, dtype=torch.float64, device=vals.device)
        buf_out = torch.empty_like(buf_in)

        def mv(x_ext, y_ext):
            ctx.bsr_spmv(vals, x_ext, y_ext)

        def pc(x_own, y_own):
            buf_in.zero_()
            buf_in[d0:d1].copy_(x_own)
            ctx.pc_apply(buf_in, buf_out, precision)
            y_own.copy_(buf_out[d0:d1])
        return cls(plan, bs, mv, pc, group)

    def _allreduce(self, t):
        import torch.distributed as dist
        if self.plan.nranks > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    def matvec(self, x_own, y_own, x_ext=None, y_ext=None):
        import torch
        x_ext = torch.zeros(self.n_ext, dtype=x_own.dtype, device=x_own.device) if x_ext is None else x_ext
        y_ext = torch.empty_like(x_ext) if y_ext is None else y_ext
        x_ext[self.d0:self.d1].copy_(x_own)
        halo_exchange(self.plan, x_ext, self.bs, self.group)
        self.local_mv(x_ext, y_ext)
        y_own.copy_(y_ext[self.d0:self.d1])

    def dots(self, V, w):
        """all-reduced V_j . w for the rows of V"""
        return self._allreduce(V @ w)

    def norm(self, v):
        import torch
        return float(torch.sqrt(self._allreduce((v @ v).reshape(1)))[0])

    def solve(self, b, x, m=30, rtol=1e-5, maxit=2000):
        """x <- J^-1 b (x holds the initial guess); returns (iterations, relative residual)"""
        import math

        import torch
        n = b.numel()
        V = torch.zeros((m + 1, n), dtype=b.dtype, device=b.device)
        Z = torch.zeros((m, n), dtype=b.dtype, device=b.device) if self.local_pc else None
        r = torch.empty_like(b)
        w = torch.empty_like(b)
        x_ext = torch.zeros(self.n_ext, dtype=b.dtype, device=b.device)
        y_ext = torch.empty_like(x_ext)
        bnorm = self.norm(b)
        if bnorm == 0.0:
            x.zero_()
            return 0, 0.0
        its = 0
        rel = 1.0
        while its < maxit:
            self.matvec(x, r, x_ext, y_ext)
            r.neg_().add_(b)
            beta = self.norm(r)
            rel = beta / bnorm
            if rel <= rtol:
                break
            V[0].copy_(r / beta)
            H = [[0.0] * m for _ in range(m + 1)]
            cs, sn = [0.0] * m, [0.0] * m
            g = [0.0] * (m + 1)
            g[0] = beta
            j = 0
            while j < m and its < maxit:
                z = V[j]
                if Z is not None:
                    self.local_pc(V[j], Z[j])
                    z = Z[j]
                self.matvec(z, w, x_ext, y_ext)
                h = self.dots(V[:j + 1], w)
                w.sub_(h @ V[:j + 1])
                h2 = self.dots(V[:j + 1], w)
                w.sub_(h2 @ V[:j + 1])
                hh = (h + h2).tolist()
                hn = self.norm(w)
                for i in range(j + 1):
                    H[i][j] = hh[i]
                H[j + 1][j] = hn
                for i in range(j):
                    t = cs[i] * H[i][j] + sn[i] * H[i + 1][j]
                    H[i + 1][j] = -sn[i] * H[i][j] + cs[i] * H[i + 1][j]
                    H[i][j] = t
                den = math.hypot(H[j][j], H[j + 1][j])
                cs[j], sn[j] = (H[j][j] / den, H[j + 1][j] / den) if den > 0 else (1.0, 0.0)
                H[j][j] = cs[j] * H[j][j] + sn[j] * H[j + 1][j]
                H[j + 1][j] = 0.0
                g[j + 1] = -sn[j] * g[j]
                g[j] = cs[j] * g[j]
                its += 1
                j += 1
                if hn > 0:
                    V[j].copy_(w / hn)
                rel = abs(g[j]) / bnorm
                if rel <= rtol or hn == 0:
                    break
            # y = H^-1 g (upper triangular), x += Z y (or V y)
            y = [0.0] * j
            for i in reversed(range(j)):
                s = g[i] - sum(H[i][k] * y[k] for k in range(i + 1, j))
                y[i] = s / H[i][i]
            basis = Z if Z is not None else V
            x.add_(torch.tensor(y, dtype=b.dtype, device=b.device) @ basis[:j])
            if rel <= rtol:
                break
        return its, rel
