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
