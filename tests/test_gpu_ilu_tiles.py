"""Block-ILU(0) on element tiles (icx_set_ilu_tile / icx_newton_options.ilu_tile).

* The apply equals a numpy restatement: block-Jacobi over s x s element tiles,
  each tile's ILU(0) in natural order (sequential IKJ block elimination on the
  tile's own blocks), then the two triangular solves, at 1e-12 of the result
  (FP64 factors) and 1e-5 (FP32 factors).
* A tile at least as large as the grid is plain ILU(0): bit-identical to the
  untiled apply with the per-tile apply that sums like the data-flow apply
  (schedule 4, the FP64 default on tiles), within 1e-14 of it with the
  one-lane-per-row apply (5, the FP32 default).
* The per-tile applies (one CTA per tile, levels in turn; matrix rows in
  registers or staged in shared memory) and the data-flow apply of the same
  tiled factors are bit-identical for every compiled rows per task, in FP64
  and FP32 factors, on ragged tiles; the one-lane-per-row apply is
  bit-identical across its CTA sizes and within 1e-13 (FP64) / 1e-5 (FP32)
  of the others.
* The preconditioner changes GMRES iterations only: Newton with tiled ILU
  reaches the untiled converged state to 1e-10 of the initial state's L2
  norm (the steady state of this Burgers problem is u = 0).
"""
import numpy as np
import pytest
import torch

from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu


def _jacobian(ctx, spec, seed=3):
    rng = np.random.default_rng(seed)
    u = torch.from_numpy(spec.state(rng)).cuda()
    L = ctx.layout
    bs = L.block_size
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    res = torch.empty_like(u)
    ctx.form_jacobian_fd(u, res, vals)
    rowptr, colidx = ctx.jacobian_pattern()
    return vals, rowptr, colidx, bs


def tiled_ilu_apply_reference(nx, ny, tile, rowptr, colidx, vals, bs, x):
    """y = M^-1 x, M = the block ILU(0) of each tile's matrix (the blocks of
    the pattern whose row and column elements lie in the same tile)"""
    E = nx * ny
    V = vals.reshape(-1, bs, bs)
    tid = [((e % nx) // tile, (e // nx) // tile) for e in range(E)]
    blocks = {}
    for r in range(E):
        for k in range(rowptr[r], rowptr[r + 1]):
            c = int(colidx[k])
            if tid[c] == tid[r]:
                blocks[(r, c)] = V[k].copy()
    # IKJ block ILU(0) in natural element order; row r's lower blocks first
    cols = {r: sorted(c for (rr, c) in blocks if rr == r) for r in range(E)}
    for r in range(E):
        for k in [c for c in cols[r] if c < r]:
            blocks[(r, k)] = blocks[(r, k)] @ np.linalg.inv(blocks[(k, k)])
            for j in [c for c in cols[k] if c > k]:
                if (r, j) in blocks:
                    blocks[(r, j)] = blocks[(r, j)] - blocks[(r, k)] @ blocks[(k, j)]
    xb = x.reshape(E, bs)
    f = np.zeros_like(xb)
    for r in range(E):
        acc = xb[r].copy()
        for k in [c for c in cols[r] if c < r]:
            acc -= blocks[(r, k)] @ f[k]
        f[r] = acc
    y = np.zeros_like(xb)
    for r in reversed(range(E)):
        acc = f[r].copy()
        for k in [c for c in cols[r] if c > r]:
            acc -= blocks[(r, k)] @ y[k]
        y[r] = np.linalg.solve(blocks[(r, r)], acc)
    return y.reshape(-1)


CASES = [
    (dict(pde=BURGERS, nx=7, ny=5, p=2), 3),
    (dict(pde=BURGERS, nx=8, ny=8, p=1, g=1), 4),
    (dict(pde=BURGERS, nx=5, ny=6, p=3), 2),
    (dict(pde=BURGERS, nx=6, ny=4, p=2), 1),        # tile 1: block-Jacobi
    (dict(pde=NS, nx=6, ny=5, p=2, ip=True), 4),    # 36 x 36 blocks, ragged last tiles
    (dict(pde=NS, nx=4, ny=4, p=3, ip=True), 2),    # 64 x 64
]


@pytest.mark.parametrize("kw,tile", CASES, ids=[f"{c}-t{t}" for c, t in CASES])
def test_tiled_apply_matches_numpy(kw, tile):
    spec = Spec(**kw)
    ctx = spec.context()
    vals, rowptr, colidx, bs = _jacobian(ctx, spec)
    ctx.ilu_tile = tile
    rng = np.random.default_rng(5)
    v = vals.cpu().numpy()
    for trial in range(2):
        x = rng.standard_normal(ctx.layout.n_dof)
        y_ref = tiled_ilu_apply_reference(spec.nx, spec.ny, tile, rowptr, colidx, v, bs, x)
        for precision, tol in ((0, 1e-12), (1, 1e-5)):
            xd = torch.from_numpy(x).cuda()
            y = torch.empty_like(xd)
            ctx.ilu_apply(vals, xd, y, precision, 1, repeat=2)
            torch.cuda.synchronize()
            err = np.abs(y.cpu().numpy() - y_ref).max()
            assert err <= tol * np.abs(y_ref).max(), (precision, err)
    ctx.close()


@pytest.mark.parametrize("kw,tile", [(dict(pde=NS, nx=13, ny=11, p=2, ip=True), 4),
                                     (dict(pde=NS, nx=9, ny=10, p=2, ip=True), 8),
                                     (dict(pde=BURGERS, nx=12, ny=7, p=3, ip=True), 5)])
def test_tile_apply_equals_data_flow_apply_bitwise(kw, tile):
    spec = Spec(**kw)
    ctx = spec.context()
    vals, _, _, _ = _jacobian(ctx, spec)
    ctx.ilu_tile = tile
    x = torch.from_numpy(np.random.default_rng(11).standard_normal(ctx.layout.n_dof)).cuda()
    bad = []
    for precision in (0, 1):
        for rows in (2, 4, 6, 8):
            ys = {}
            # data flow; per-tile applies in registers / staged, 512 / 256 / 128 threads per CTA
            for sched, k in ((2, 0), (4, 0), (3, 0), (4, 1), (4, 2), (4, 3), (3, 1), (3, 3),
                             (5, 0), (5, 1), (5, 2), (5, 3)):
                ctx.tile = {"ilu_sched": [sched, sched], "ilu_rows": [rows, rows], "ilu_ctas": [k, k]}
                y = torch.full_like(x, float("nan"))
                ctx.ilu_apply(vals, x, y, precision, 1, repeat=2)
                ys[(sched, k)] = y
            torch.cuda.synchronize()
            y0 = ys.pop((2, 0))
            assert torch.isfinite(y0).all()
            for key, y in ys.items():
                ref = ys[(5, 0)] if key[0] == 5 else y0
                if not torch.equal(ref.view(torch.int64), y.view(torch.int64)):
                    d = (y - ref).abs()
                    bad.append((precision, rows, key, int((d > 0).sum()), float(d.max())))
            tol = 1e-13 if precision == 0 else 1e-5
            assert float((ys[(5, 0)] - y0).abs().max()) <= tol * float(y0.abs().max()), (precision, rows)
    assert not bad, bad
    ctx.tile = {}
    ctx.close()


def test_tile_covering_grid_is_plain_ilu():
    spec = Spec(pde=NS, nx=6, ny=5, p=2, ip=True)
    ctx = spec.context()
    vals, _, _, _ = _jacobian(ctx, spec)
    x = torch.from_numpy(np.random.default_rng(9).standard_normal(ctx.layout.n_dof)).cuda()
    y0, y1 = torch.empty_like(x), torch.empty_like(x)
    y5 = torch.empty_like(x)
    ctx.ilu_tile = 0
    ctx.ilu_apply(vals, x, y0, 0, 1)
    ctx.ilu_tile = 8
    ctx.ilu_apply(vals, x, y1, 0, 1)
    ctx.tile = {"ilu_sched": [5, 5]}
    ctx.ilu_apply(vals, x, y5, 0, 1)
    ctx.tile = {}
    torch.cuda.synchronize()
    assert torch.equal(y0.view(torch.int64), y1.view(torch.int64))
    assert float((y5 - y0).abs().max()) <= 1e-14 * float(y0.abs().max())
    ctx.close()


@pytest.mark.parametrize("tile", [4, 8])
def test_newton_with_tiled_ilu_reaches_same_state(tile):
    import iceicle_b200 as ib
    from iceicle_b200.workloads import burgers_config
    wl = burgers_config(nx=24, ny=24)
    out = {}
    for t in (0, tile):
        for prec in (0, 1):
            o = ib.default_newton_options()
            o.ilu_tile, o.precision, o.gmres_rtol = t, prec, 1e-8
            u = torch.from_numpy(wl.u0.copy()).cuda()
            rep = wl.ctx.newton_solve(u, o)
            assert rep.converged
            out[(t, prec)] = (u.cpu().numpy(), rep.linear_iterations_total)
    base = out[(0, 0)][0]
    scale = max(np.linalg.norm(base), np.linalg.norm(wl.u0))
    for key, (u, _) in out.items():
        assert np.linalg.norm(u - base) <= 1e-10 * scale, key


def test_element_groups_and_separate_factor_apply():
    """icx_set_ilu_groups + icx_pc_factor / icx_pc_apply: groups equal to the
    2 x 2 tiles give the tiled apply bit for bit; one group holding every
    element is the whole grid's ILU(0)"""
    spec = Spec(pde=NS, nx=6, ny=5, p=2, ip=True)
    ctx = spec.context()
    vals, _, _, _ = _jacobian(ctx, spec)
    x = torch.from_numpy(np.random.default_rng(2).standard_normal(ctx.layout.n_dof)).cuda()
    y_tile, y_grp, y_all, y_nat = (torch.empty_like(x) for _ in range(4))
    ctx.ilu_tile = 2
    ctx.ilu_apply(vals, x, y_tile, 0, 1)
    ctx.ilu_tile = 0
    e = np.arange(30)
    ctx.set_ilu_groups((e % 6) // 2 + 3 * ((e // 6) // 2))
    ctx.pc_factor(vals, 0)
    ctx.pc_apply(x, y_grp, 0)
    ctx.set_ilu_groups(np.zeros(30))
    ctx.pc_factor(vals, 0)
    ctx.pc_apply(x, y_all, 0)
    ctx.set_ilu_groups(None)
    ctx.ilu_apply(vals, x, y_nat, 0, 1)
    torch.cuda.synchronize()
    assert torch.equal(y_tile.view(torch.int64), y_grp.view(torch.int64))
    assert float((y_all - y_nat).abs().max()) <= 1e-12 * float(y_nat.abs().max())
    ctx.close()


def test_strip_krylov_on_one_rank_matches_gmres():
    """the partitioned GMRES (iceicle_b200.partition.StripKrylov) over a GPU
    context with one rank: BSR product and the owned-block ILU(0) through
    icx_pc_factor / icx_pc_apply; the solution equals icx_gmres_solve's"""
    from iceicle_b200.partition import StripKrylov, StripPlan
    spec = Spec(pde=NS, nx=8, ny=8, p=2, ip=True)
    ctx = spec.context()
    vals, _, _, _ = _jacobian(ctx, spec)
    b = torch.from_numpy(np.random.default_rng(6).standard_normal(ctx.layout.n_dof)).cuda()
    plan = StripPlan(spec.nx, spec.ny, 1, 0, spec.g)
    kry = StripKrylov.for_context(ctx, plan, vals)
    x = torch.zeros_like(b)
    its, rel = kry.solve(b, x, m=30, rtol=1e-12, maxit=5000)
    ctx.set_ilu_groups(None)
    x2 = torch.zeros_like(b)
    ctx.gmres_solve(vals, b, x2, restart=30, maxit=5000, rtol=1e-12, preconditioner=2)
    torch.cuda.synchronize()
    assert rel <= 1e-12
    assert float((x - x2).norm() / x2.norm()) <= 1e-9
    ctx.close()


@pytest.mark.parametrize("kw,tile", [(dict(pde=NS, nx=13, ny=11, p=2, ip=True), 4),
                                     (dict(pde=BURGERS, nx=12, ny=7, p=3, ip=True), 5)])
def test_bf16_factors_apply(kw, tile):
    """precision 2 of icx_ilu_apply: the tiled factors rounded to BF16, widened
    to FP32 in the one-lane-per-row apply. Against the FP64 apply of the same
    factors the result differs by the factors' rounding (2^-9 relative per
    value): within 5e-2 of the result's largest entry, and identical across
    CTA sizes"""
    spec = Spec(**kw)
    ctx = spec.context()
    vals, _, _, _ = _jacobian(ctx, spec)
    ctx.ilu_tile = tile
    x = torch.from_numpy(np.random.default_rng(12).standard_normal(ctx.layout.n_dof)).cuda()
    y64 = torch.empty_like(x)
    ctx.ilu_apply(vals, x, y64, 0, 1)
    ys = []
    for k in (0, 1, 2, 3):
        ctx.tile = {"ilu_sched": [5, 5], "ilu_ctas": [k, k]}
        y = torch.full_like(x, float("nan"))
        ctx.ilu_apply(vals, x, y, 2, 1, repeat=2)
        ys.append(y)
    ctx.tile = {}
    torch.cuda.synchronize()
    assert torch.isfinite(ys[0]).all()
    for y in ys[1:]:
        assert torch.equal(ys[0].view(torch.int64), y.view(torch.int64))
    err = float((ys[0] - y64).abs().max()) / float(y64.abs().max())
    assert err <= 5e-2, err
    ctx.close()
