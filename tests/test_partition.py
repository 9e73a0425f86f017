"""Element-row partitioning and the halo exchange (iceicle_b200.partition),
on the CPU: the plan's rows, nodes and DOF ranges; and, with gloo ranks in
separate processes, the exchange of boundary rows followed by the oracle
residual of every rank's sub-mesh, whose owned entries must equal the global
oracle residual exactly (the partition of form_residual.hpp:87-135)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from iceicle_b200.partition import StripPlan, strip_rows, sub_coords


@pytest.mark.parametrize("ny,nranks", [(7, 1), (7, 2), (7, 3), (8, 4), (9, 9), (128, 8)])
def test_strip_rows_cover_and_balance(ny, nranks):
    rows = [strip_rows(ny, nranks, r) for r in range(nranks)]
    assert rows[0][0] == 0 and rows[-1][1] == ny
    for (a0, a1), (b0, b1) in zip(rows, rows[1:]):
        assert a1 == b0
    sizes = [b - a for a, b in rows]
    assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


def test_strip_rows_refuses_too_many_ranks():
    with pytest.raises(ValueError):
        strip_rows(3, 4, 0)


@pytest.mark.parametrize("nranks", [1, 2, 3, 7])  # 7: one owned row per rank
def test_plan_ranges(nranks):
    nx, ny, g, bs = 5, 7, 2, 36
    for r in range(nranks):
        p = StripPlan(nx, ny, nranks, r, g)
        assert p.g0 == (p.j0 - 1 if r > 0 else 0) and p.g1 == (p.j1 + 1 if r < nranks - 1 else ny)
        e0, e1 = p.owned_elements()
        assert e1 - e0 == (p.j1 - p.j0) * nx and e0 == (p.j0 - p.g0) * nx
        n0, n1 = p.node_range()
        w = nx * g + 1
        assert (n1 - n0) == (p.rows * g + 1) * w and n0 == p.g0 * g * w
        d0, d1 = p.global_dofs(bs)
        assert d1 - d0 == p.rows * nx * bs
        # the halo: what a rank sends to a neighbour is what that neighbour receives
        for peer, (s0, s1), (r0, r1) in p.halo(bs):
            q = StripPlan(nx, ny, nranks, peer, g)
            back = [h for h in q.halo(bs) if h[0] == r][0]
            # global row indices of the sent row and of the row the peer receives
            sent_row = p.g0 + s0 // (nx * bs)
            recv_row_at_peer = q.g0 + back[2][0] // (nx * bs)
            assert sent_row == recv_row_at_peer
            assert s1 - s0 == r1 - r0 == nx * bs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, nranks, port, kw, q):
    """one gloo rank: its sub-mesh state with the ghost rows set to NaN, the
    exchange, then the oracle residual of the sub-mesh against the global one"""
    try:
        import torch
        import torch.distributed as dist

        import oracle_bindings as ob
        from iceicle_b200.partition import halo_exchange
        from specs import Spec
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=nranks,
                                timeout=__import__("datetime").timedelta(seconds=60))
        spec = Spec(**kw)
        c = spec.coords()
        u = spec.state(np.random.default_rng(9))
        bs = spec.nb * spec.neq
        r_glob = ob.residual(ob.oracle(), spec.oracle_problem(), c, u)
        plan = StripPlan(spec.nx, spec.ny, nranks, rank, spec.g)
        d0, d1 = plan.global_dofs(bs)
        ul = torch.from_numpy(u[d0:d1].copy())
        # ghost rows come only from the exchange
        ghost = np.ones(d1 - d0, dtype=bool)
        o0, o1 = plan.owned_dofs(bs)
        ghost[o0:o1] = False
        ul[torch.from_numpy(ghost)] = float("nan")
        n = halo_exchange(plan, ul, bs)
        assert n == int(ghost.sum()), (n, int(ghost.sum()))
        assert np.array_equal(ul.numpy(), u[d0:d1]), "ghost rows after the exchange"
        sub = Spec(**dict(kw, ny=plan.rows))
        r_sub = ob.residual(ob.oracle(), sub.oracle_problem(), sub_coords(plan, c), ul.numpy())
        e0, e1 = plan.owned_elements()
        mine = r_sub[e0 * bs:e1 * bs]
        ref = r_glob[(plan.j0 * spec.nx) * bs:(plan.j1 * spec.nx) * bs]
        assert np.array_equal(mine, ref), float(np.abs(mine - ref).max())
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except BaseException as e:  # reported to the parent
        q.put((rank, repr(e)))


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("kw", [dict(pde=0, nx=4, ny=6, p=2), dict(pde=1, nx=3, ny=5, p=2, ip=True, source=True)],
                         ids=["burgers_ddg", "ns_ip"])
def test_gloo_halo_exchange_and_partitioned_residual(nranks, kw):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, nranks, port, kw, q)) for r in range(nranks)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(nranks):
            r, msg = q.get(timeout=240)
            out[r] = msg
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    assert out == {r: "ok" for r in range(nranks)}, out
