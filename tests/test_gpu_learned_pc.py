"""The learned block preconditioner (Newton preconditioner 5) and the
parallel preconditioners 3 and 4: the BF16 graph network (MLP with one
face-neighbour message-passing step) against a torch FP32 evaluation of the
same network on BF16-rounded inputs, training lowering its loss, and Newton
solves that reach the plain block-ILU(0) state."""
import numpy as np
import pytest
import torch

import iceicle_b200 as ib
from specs import NS, Spec

pytestmark = pytest.mark.gpu


def _ns_ctx(nx=6, ny=5):
    spec = Spec(pde=NS, nx=nx, ny=ny, g=2, p=2, ip=True, source=True, perturb=0.05)
    ctx = spec.context()
    from test_gpu_solver import _ns_mms_state
    u0 = _ns_mms_state(ctx, 1e-2, 5)
    return spec, ctx, u0


def _jacobian(ctx, u):
    L = ctx.layout
    bs = L.block_size
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
    res = torch.empty_like(u)
    ctx.form_jacobian_fd(u, res, vals)
    return vals, res


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


def test_mlp_forward_matches_a_torch_fp32_evaluation():
    """h1_e = relu(W1 x_e + b1), m_e = mean of h1 over the face neighbours of e
    (the message-passing step), h2_e = relu(W2 [h1_e ; m_e] + b2),
    C_e = W3 h2_e + b3, x_e = J_ee / |J_ee|_F. The reference rounds x, the
    weights, h1, m and h2 to BF16 as the kernels do and computes in FP32; the
    kernels accumulate in FP32 in another order: 2e-2 of the largest output
    (BF16 has 8 bits)."""
    spec, ctx, u0 = _ns_ctx()
    m = ib.LearnedPreconditioner(36, 64, 0, seed=3)
    p = m.get_params()
    rng = np.random.default_rng(0)
    D, H = 36 * 36, 64
    oW2 = H * D + H
    oW3 = oW2 + H * 2 * H + H
    assert p.size == oW3 + D * H + D
    p[oW3:oW3 + D * H] = 0.05 * rng.standard_normal(D * H)
    p[oW3 + D * H:] = 0.01 * rng.standard_normal(D)
    p[H * D:H * D + H] = 0.1 * rng.standard_normal(H)
    m.set_params(p)
    ctx.lpc_attach(m)
    u = torch.from_numpy(u0).cuda()
    vals, _ = _jacobian(ctx, u)
    E = ctx.layout.n_elem
    corr = torch.empty(E * D, dtype=torch.float32, device="cuda")
    ctx.lpc_forward(vals, corr)
    torch.cuda.synchronize()
    rp, ci = ctx.jacobian_pattern()
    diag = np.array([rp[e] + int(np.nonzero(ci[rp[e]:rp[e + 1]] == e)[0][0]) for e in range(E)])
    V = vals.view(-1, D)[torch.from_numpy(diag).cuda()]
    X = _bf((V / V.norm(dim=1, keepdim=True)).float())
    P = torch.from_numpy(p).cuda()
    W1 = P[:H * D].view(H, D); b1 = P[H * D:oW2]
    W2 = P[oW2:oW2 + 2 * H * H].view(H, 2 * H); b2 = P[oW2 + 2 * H * H:oW3]
    W3 = P[oW3:oW3 + D * H].view(D, H); b3 = P[oW3 + D * H:]
    h1 = _bf(torch.relu(X @ _bf(W1).T + b1))
    msg = torch.zeros_like(h1)
    for e in range(E):
        nb = [int(k) for k in ci[rp[e]:rp[e + 1]] if k != e]
        if nb:
            msg[e] = h1[nb].mean(dim=0)
    h2 = _bf(torch.relu(torch.cat([h1, _bf(msg)], dim=1) @ _bf(W2).T + b2))
    ref = h2 @ _bf(W3).T + b3
    got = corr.view(E, D)
    assert (got - ref).abs().max().item() <= 2e-2 * ref.abs().max().item()
    # the message matters: the same network without it gives another output
    h2_nomsg = _bf(torch.relu(torch.cat([h1, torch.zeros_like(h1)], dim=1) @ _bf(W2).T + b2))
    ref_nomsg = h2_nomsg @ _bf(W3).T + b3
    assert (ref_nomsg - ref).abs().max().item() > 5e-2 * ref.abs().max().item()
    ctx.lpc_attach(None)


def test_training_lowers_the_preconditioned_residual():
    """Adam steps on Krylov residuals of one Jacobian lower the mean of
    |r - J (I + C) ILU_1(r)|^2 / |r|^2 (first loss: the untrained model, C = 0)"""
    spec, ctx, u0 = _ns_ctx()
    m = ib.LearnedPreconditioner(36, 64, 0, seed=1)
    ctx.lpc_attach(m)
    u = torch.from_numpy(u0).cuda()
    vals, res = _jacobian(ctx, u)
    buf = torch.empty((48, ctx.layout.n_dof), dtype=torch.float64, device="cuda")
    du = torch.empty_like(u)
    ns, its, rr = ctx.krylov_samples(vals, res, du, buf, every=2, rtol=1e-8)
    assert ns >= 8
    rep = ctx.lpc_train(vals, buf, ns, steps=60, batch=4, sweeps=1, lr=2e-3, seed=2)
    hist = list(rep.loss_history[:60])
    assert np.isfinite(hist).all()
    assert np.mean(hist[-10:]) < 0.9 * np.mean(hist[:5]), hist
    assert m.steps == 60
    ctx.lpc_attach(None)


def test_calibration_sums_and_scaling():
    """icx_lpc_calibrate after a few training steps: positive sums, the loss
    at the chosen g is the clamped quadratic optimum (no worse than the base
    preconditioner, g = 0, or the full correction, g = 1), and scaling the
    output layer by a power of two scales the correction by it exactly"""
    spec, ctx, u0 = _ns_ctx()
    m = ib.LearnedPreconditioner(36, 64, 0, seed=4)
    ctx.lpc_attach(m)
    u = torch.from_numpy(u0).cuda()
    vals, res = _jacobian(ctx, u)
    buf = torch.empty((24, ctx.layout.n_dof), dtype=torch.float64, device="cuda")
    du = torch.empty_like(u)
    ns, _, _ = ctx.krylov_samples(vals, res, du, buf, every=2, rtol=1e-8)
    ctx.lpc_train(vals, buf, ns, steps=30, batch=4, sweeps=0, lr=2e-3, seed=5)
    ab, bb, aa = ctx.lpc_calibrate(vals, buf, ns, 0)
    assert bb > 0 and aa > 0
    g = min(max(ab / bb, 0.0), 1.0)
    q = lambda t: aa - 2 * t * ab + t * t * bb
    assert q(g) <= min(q(0.0), q(1.0)) * (1 + 1e-12)
    E, D = ctx.layout.n_elem, 36 * 36
    c0 = torch.empty(E * D, dtype=torch.float32, device="cuda")
    ctx.lpc_forward(vals, c0)
    p = m.get_params()
    o_w3 = 64 * D + 64 + 64 * 128 + 64
    p[o_w3:] *= 0.5
    m.set_params(p)
    c1 = torch.empty_like(c0)
    ctx.lpc_forward(vals, c1)
    torch.cuda.synchronize()
    # BF16 rounding of W3 is exact under a scale by 1/2
    assert torch.allclose(c1, 0.5 * c0, rtol=0, atol=1e-6 * float(c0.abs().max()))
    ctx.lpc_attach(None)


@pytest.mark.parametrize("pc,prec,sweeps", [(3, 0, 0), (4, 0, 1), (4, 1, 2), (5, 1, 1), (5, 0, 2)])
def test_parallel_and_learned_preconditioners_reach_the_ilu0_state(pc, prec, sweeps):
    """the Newton solve with preconditioner pc converges to the state of the
    plain FP64 block-ILU(0) solve (both to |r| <= 1e-10; states to 1e-9,
    relative L2) without falling back"""
    spec, ctx, u0 = _ns_ctx()
    m = ib.LearnedPreconditioner(36, 64, 0, seed=4)
    if pc == 5:
        ctx.lpc_attach(m)
    o = ib.default_newton_options()
    o.gmres_max_it = 5000
    u1 = torch.from_numpy(u0.copy()).cuda()
    r1 = ctx.newton_solve(u1, o)
    o2 = ib.default_newton_options()
    o2.gmres_max_it = 5000
    o2.preconditioner, o2.precision, o2.pc_sweeps = pc, prec, sweeps
    u2 = torch.from_numpy(u0.copy()).cuda()
    r2 = ctx.newton_solve(u2, o2)
    assert r1.converged and r2.converged
    assert r2.pc_fallbacks == 0
    a, b = u1.cpu().numpy(), u2.cpu().numpy()
    assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(a)
    ctx.lpc_attach(None)


def test_missed_linear_tolerance_falls_back_to_ilu0():
    spec, ctx, u0 = _ns_ctx()
    o = ib.default_newton_options()
    o.preconditioner, o.gmres_max_it, o.kmax = 3, 3, 2
    u = torch.from_numpy(u0.copy()).cuda()
    rep = ctx.newton_solve(u, o)
    assert rep.pc_fallbacks >= 1


def test_learned_preconditioner_needs_a_model():
    spec, ctx, u0 = _ns_ctx(3, 3)
    o = ib.default_newton_options()
    o.preconditioner = 5
    with pytest.raises(ib.IcxError):
        ctx.newton_solve(torch.from_numpy(u0.copy()).cuda(), o)
    m = ib.LearnedPreconditioner(16, 64, 0)
    with pytest.raises(ib.IcxError):
        ctx.lpc_attach(m)  # block size 16 on a 36 x 36 block context


def test_model_save_and_load(tmp_path):
    m = ib.LearnedPreconditioner(36, 64, 0, seed=9)
    p = m.get_params()
    p += np.random.default_rng(1).standard_normal(p.size).astype(np.float32) * 1e-3
    m.set_params(p)
    m.save(tmp_path / "m.npz")
    m2 = ib.LearnedPreconditioner.load(tmp_path / "m.npz")
    assert np.array_equal(m2.get_params(), p)


@pytest.mark.parametrize("prec,tile", [(1, 0), (1, 2), (0, 0)])
def test_zero_output_layer_is_its_base_preconditioner(prec, tile):
    """a model whose output layer (W3, b3) is zero has C = 0: preconditioner 5
    is then its base (block-ILU(0), sweeps = 0) without the network's
    products, and the Newton solve is the base's bit for bit (iterations,
    GMRES counts, state), its Arnoldi steps replayed as graphs"""
    from iceicle_b200 import learned_pc as lp
    spec, ctx, u0 = _ns_ctx()
    m = ib.LearnedPreconditioner(36, 64, 0, seed=4)
    p = m.get_params()
    D, H = 36 * 36, 64
    p[H * D + H + H * 2 * H + H:] = 0
    m.set_params(p)
    assert lp.correction_is_zero(m)
    out = {}
    for pc in (2, 5):
        ctx.lpc_attach(m if pc == 5 else None)
        o = ib.default_newton_options()
        o.gmres_max_it, o.preconditioner, o.precision, o.pc_sweeps, o.ilu_tile = 5000, pc, prec, 0, tile
        u = torch.from_numpy(u0.copy()).cuda()
        r = ctx.newton_solve(u, o)
        assert r.converged
        out[pc] = (u.cpu().numpy(), r.iterations, list(r.linear_iterations[:r.iterations]), r.graph_steps)
    ctx.lpc_attach(None)
    (a, ia, la, ga), (b, ib_, lb, gb) = out[2], out[5]
    assert ia == ib_ and la == lb and gb > 0
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
