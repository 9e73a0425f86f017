"""The partitioned linear solve of a Newton step (iceicle_b200.partition.
StripKrylov) on gloo ranks in separate processes, CPU only: each rank holds
the block rows of its element-row strip of the oracle's FD Jacobian (owned
rows, columns of its ghost rows), multiplies after the halo exchange of the
vector's boundary rows, all-reduces its Gram-Schmidt coefficients, and
preconditions with the ILU(0) of its owned block (block-Jacobi across ranks,
PETSc's parallel default). Checked against the global system:

* the partitioned product equals the global product on every owned row
  (the same sums in the same order: exactly);
* GMRES to 1e-11 reaches the global sparse direct solution to 1e-8;
* with one rank the preconditioner is the whole grid's ILU(0), and GMRES
  needs fewer iterations than with three ranks (the dropped couplings cost
  iterations, not accuracy)."""
import multiprocessing as mp
import os

import numpy as np
import pytest

from iceicle_b200.partition import StripPlan
from test_partition import _free_port


def block_ilu0(blocks, n):
    """IKJ block ILU(0) of {(r, c): block} over elements 0..n-1 in natural
    order (the blocks present are the pattern); returns a solver x -> M^-1 x"""
    B = {k: v.copy() for k, v in blocks.items()}
    cols = {r: sorted(c for (rr, c) in B if rr == r) for r in range(n)}
    for r in range(n):
        for k in [c for c in cols[r] if c < r]:
            B[(r, k)] = B[(r, k)] @ np.linalg.inv(B[(k, k)])
            for j in [c for c in cols[k] if c > k]:
                if (r, j) in B:
                    B[(r, j)] = B[(r, j)] - B[(r, k)] @ B[(k, j)]
    bs = next(iter(B.values())).shape[0]

    def solve(x):
        xb = np.asarray(x).reshape(n, bs)
        f = np.zeros_like(xb)
        for r in range(n):
            f[r] = xb[r] - sum((B[(r, k)] @ f[k] for k in cols[r] if k < r), np.zeros(bs))
        y = np.zeros_like(xb)
        for r in reversed(range(n)):
            acc = f[r] - sum((B[(r, k)] @ y[k] for k in cols[r] if k > r), np.zeros(bs))
            y[r] = np.linalg.solve(B[(r, r)], acc)
        return y.reshape(-1)
    return solve


def _rank_main(rank, nranks, port, kw, q):
    try:
        import scipy.sparse as sp
        import scipy.sparse.linalg as spla
        import torch
        import torch.distributed as dist

        import oracle_bindings as ob
        from iceicle_b200.partition import StripKrylov
        from specs import Spec
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=nranks,
                                timeout=__import__("datetime").timedelta(seconds=60))
        torch.set_default_dtype(torch.float64)
        spec = Spec(**kw)
        c = spec.coords()
        u = spec.state(np.random.default_rng(9))
        r_glob, rowptr, colidx, vals = ob.jacobian_bsr(spec.oracle_problem(), c, u)
        bs = vals.shape[1]
        N = u.size
        Jg = sp.bsr_matrix((vals, colidx, rowptr), shape=(N, N)).tocsr()
        plan = StripPlan(spec.nx, spec.ny, nranks, rank, spec.g)
        ge0 = plan.g0 * spec.nx                  # first element of the sub-mesh
        e0, e1 = plan.owned_elements()           # owned, sub-mesh numbering
        ne_sub = plan.rows * spec.nx
        # the rank's block rows on the sub-mesh vector: owned rows, ghost rows zero
        J_loc = Jg[(ge0 + e0) * bs:(ge0 + e1) * bs, ge0 * bs:(ge0 + ne_sub) * bs]
        d0, d1 = plan.owned_dofs(bs)

        def mv(x_ext, y_ext):
            y_ext.zero_()
            y_ext[d0:d1] = torch.from_numpy(J_loc @ x_ext.numpy())
        # block-Jacobi across ranks: ILU(0) of the owned block
        own = {}
        for r in range(e0, e1):
            gr = ge0 + r
            for k in range(rowptr[gr], rowptr[gr + 1]):
                gc = colidx[k] - ge0
                if e0 <= gc < e1:
                    own[(r - e0, gc - e0)] = vals[k]
        solve = block_ilu0(own, e1 - e0)

        def pc(x_own, y_own):
            y_own.copy_(torch.from_numpy(solve(x_own.numpy())))
        kry = StripKrylov(plan, bs, mv, pc)
        # products
        rng = np.random.default_rng(4)
        xg = rng.standard_normal(N)
        go0, go1 = (ge0 + e0) * bs, (ge0 + e1) * bs
        y = torch.empty(d1 - d0)
        kry.matvec(torch.from_numpy(xg[go0:go1].copy()), y)
        assert np.array_equal(y.numpy(), (Jg @ xg)[go0:go1])
        # solve
        x = torch.zeros(d1 - d0)
        its, rel = kry.solve(torch.from_numpy(r_glob[go0:go1].copy()), x, m=30, rtol=1e-11, maxit=3000)
        ref = spla.spsolve(Jg.tocsc(), r_glob)
        err = np.linalg.norm(x.numpy() - ref[go0:go1]) / np.linalg.norm(ref)
        assert rel <= 1e-11 and err <= 1e-8, (its, rel, err)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ("ok", its)))
    except BaseException as e:  # reported to the parent
        q.put((rank, (repr(e), -1)))


def _run(nranks, kw):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, nranks, port, kw, q)) for r in range(nranks)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(nranks):
            r, msg = q.get(timeout=300)
            out[r] = msg
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    assert all(m[0] == "ok" for m in out.values()), out
    its = {m[1] for m in out.values()}
    assert len(its) == 1, out  # every rank took the same iterations
    return its.pop()


@pytest.mark.parametrize("kw", [dict(pde=0, nx=5, ny=6, p=2), dict(pde=1, nx=3, ny=6, p=1, g=1, ip=True)],
                         ids=["burgers", "ns"])
def test_gloo_partitioned_gmres(kw):
    its1 = _run(1, kw)
    its3 = _run(3, kw)
    assert its1 <= its3, (its1, its3)
