"""The launch-shape autotuner: every compiled shape of the face, volume and
data-flow ILU kernels gives results bit-identical to the default shape's; the
tuned context still matches the oracle; choices are cached per
(dim, p, neq, geometry order, flux) and reused untimed; shapes that are not
compiled are refused."""
import numpy as np
import pytest
import torch

import iceicle_b200 as icx
import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.gpu

VOL_TILES = [(0, 0), (256, 4), (256, 3), (128, 8), (128, 6)]

CASES = [
    dict(pde=BURGERS, nx=6, ny=5, p=2),                 # 9 x 9 blocks, DDG
    dict(pde=BURGERS, nx=5, ny=4, p=4, g=1),            # 25 x 25
    dict(pde=NS, nx=5, ny=4, p=2, ip=True),             # 36 x 36, interior penalty
    dict(pde=NS, nx=4, ny=3, p=3),                      # 64 x 64, DDG (face bound 3)
]


def _setup(kw):
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(5))
    ctx = spec.context(c)
    return spec, c, u, ctx


def _residual(ctx, du):
    r = torch.full_like(du, float("nan"))
    ctx.form_residual(du, r)
    torch.cuda.synchronize()
    return r.cpu().numpy()


@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
def test_residual_shapes_bit_identical(kw):
    spec, c, u, ctx = _setup(kw)
    du = torch.from_numpy(u).cuda()
    ref = _residual(ctx, du)
    d = 3 if (kw["pde"] == NS and not kw.get("ip")) else 5
    for fm in (0, d - 1, d, d + 1):
        for vt, vm in VOL_TILES:
            ctx.tile = {"face_minb": fm, "vol_threads": vt, "vol_minb": vm}
            r = _residual(ctx, du)
            assert np.array_equal(r.view(np.uint64), ref.view(np.uint64)), (fm, vt, vm)


@pytest.mark.parametrize("kw", CASES, ids=[str(c) for c in CASES])
def test_ilu_shapes_bit_identical(kw):
    spec, c, u, ctx = _setup(kw)
    du = torch.from_numpy(u).cuda()
    L = ctx.layout
    bs = L.block_size
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    ctx.form_jacobian_fd(du, torch.empty_like(du), vals)
    x = torch.from_numpy(np.random.default_rng(8).standard_normal(L.n_dof)).cuda()
    ns = (bs + 31) // 32
    rows = [r for r in (2, 4, 6, 8) if r <= max(bs, 2) and r * ns <= 24]
    for precision in (0, 1):
        ctx.tile = {}
        y0 = torch.empty_like(x)
        ctx.ilu_apply(vals, x, y0, precision, 0)
        for sched in (1, 2):  # completion counters, sentinel values
            for r in rows:
                for k in (1, 2, 3, 4):
                    t = {"ilu_rows": [0, 0], "ilu_ctas": [0, 0], "ilu_sched": [0, 0]}
                    t["ilu_rows"][precision] = r
                    t["ilu_ctas"][precision] = k
                    t["ilu_sched"][precision] = sched
                    ctx.tile = t
                    y = torch.empty_like(x)
                    ctx.ilu_apply(vals, x, y, precision, 0, repeat=2)
                    torch.cuda.synchronize()
                    assert torch.equal(y.view(torch.int64), y0.view(torch.int64)), (precision, sched, r, k)


def test_autotune_parity_and_cache():
    kw = dict(pde=NS, nx=6, ny=5, p=2, ip=True)
    spec, c, u, ctx = _setup(kw)
    du = torch.from_numpy(u).cuda()
    rep = ctx.autotune(du, icx.TUNE_RESIDUAL | icx.TUNE_ILU | icx.TUNE_ILU_FP32 | icx.TUNE_RETIME)
    assert rep["from_cache"] == 0 and rep["n_rejected"] == 0
    # residual: the default, two face bounds, three volume tiles; ILU, per
    # precision: 2 schedules x rows 2/4/6/8 x CTAs per SM 1..4 (36 x 36 blocks)
    assert rep["n_timed"] == 6 + 2 * 32
    assert rep["residual_ms_tuned"] <= rep["residual_ms_default"]
    for k in range(2):
        assert 0 < rep["ilu_ms_tuned"][k] <= rep["ilu_ms_default"][k]
    ch = rep["chosen"]
    assert ch == ctx.tile
    assert ch["face_minb"] in (4, 5, 6)
    assert (ch["vol_threads"], ch["vol_minb"]) in VOL_TILES[1:]
    assert all(r in (2, 4, 6, 8) for r in ch["ilu_rows"]) and all(1 <= k <= 4 for k in ch["ilu_ctas"])
    assert all(sc in (1, 2) for sc in ch["ilu_sched"])
    # the tuned residual is still the reference's residual
    r_or = ob.residual(ob.oracle(), spec.oracle_problem(), c, u)
    r = _residual(ctx, du)
    assert np.abs(r - r_or).max() <= 1e-12 * np.abs(r_or).max()
    # a second context with the same key takes the cached choice untimed
    ctx2 = Spec(**kw).context(c)
    rep2 = ctx2.autotune(du)
    assert rep2["from_cache"] == 7 and rep2["n_timed"] == 0
    assert ctx2.tile == ch


def test_tile_set_refuses_uncompiled_shapes():
    spec, c, u, ctx = _setup(dict(pde=BURGERS, nx=3, ny=3, p=1, g=1))  # 4 x 4 blocks: rows 2 and 4 only
    bad = [{"face_minb": 2}, {"face_minb": 7}, {"vol_threads": 128, "vol_minb": 4}, {"vol_threads": 512},
           {"ilu_rows": [6, 0]}, {"ilu_rows": [0, 3]}, {"ilu_ctas": [5, 0]}, {"ilu_ctas": [0, -1]},
           {"ilu_sched": [6, 0]}, {"ilu_sched": [0, -1]}, {"ilu_sched": [5, 0], "ilu_ctas": [4, 0]}]
    for t in bad:
        with pytest.raises(icx.IcxError):
            ctx.tile = t
    assert ctx.tile == icx.TileChoice().as_dict()
    du = torch.from_numpy(u).cuda()
    with pytest.raises(icx.IcxError):
        ctx.autotune(du, 16)
