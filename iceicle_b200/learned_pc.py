"""Training and evaluation of the learned block preconditioner (Newton
preconditioner 5) on the 2D compressible Navier-Stokes manufactured solution:
n x n quadrilaterals on [0,1]^2 with geometry order 2, p = 2 (9 basis
functions x 4 conserved variables: 36 x 36 Jacobian blocks), Van Leer flux
with interior penalty, nodes perturbed by a seeded smooth displacement, and a
Reynolds number drawn per instance uniformly from [50, 500] (viscosity 1/Re).

Training data are generated by the solver the correction is trained for: at
every Newton step of a training instance the FD Jacobian is formed and the
GMRES(30) solve of that step with the base preconditioner (block-ILU(0) on
element tiles) records Krylov residuals (its restart residuals and every
k-th Arnoldi vector); each (Jacobian, residual) pair is one training sample,
and instances are drawn until the recipe's number of pairs is reached. The model then takes Adam steps on that Jacobian's samples
before the Newton step is applied. The correction is trained on top of the
base preconditioner it is run with (block-ILU(0) on element tiles, exact
triangular solves). Evaluation runs fresh seeds through the plain all-FP64
block-ILU(0) Newton solve and through the learned, mixed-precision one, both
to an FP64 residual of 1e-10."""
import time

import numpy as np

from . import LearnedPreconditioner, default_newton_options
from .workloads import ns_mms_config

BLOCK_SIZE = 36


def instances(n, seed, re_range=(50.0, 500.0)):
    """n seeded (mesh and state seed, Reynolds number) pairs"""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(1, 2**31 - 1)), float(rng.uniform(*re_range))) for _ in range(n)]


def make_instance(seed, re, n=256, device=0):
    return ns_mms_config(nx=n, ny=n, p=2, geo_order=2, seed=seed, device=device, mu=1.0 / re)


def train(model, train_instances, n=256, samples=167, every=10, steps=150, batch=4, random=2, sweeps=2, lr=1e-3,
          newton_steps=4, device=0, log=None, pairs=None, ilu_tile=0):
    """train `model` on the Newton steps of each instance (until `pairs`
    Jacobian / residual pairs have been used, when given); returns
    per-Jacobian records (instance, step, |r|, samples, gmres iterations,
    first/last loss)"""
    import torch
    dev = torch.device("cuda", device)
    out = []
    used = 0
    for (seed, re) in train_instances:
        if pairs is not None and used >= pairs:
            break
        wl = make_instance(seed, re, n, device)
        ctx = wl.ctx
        ctx.ilu_tile = ilu_tile
        ctx.lpc_attach(model)
        L = ctx.layout
        bs = L.block_size
        u = torch.from_numpy(wl.u0).to(dev)
        res = torch.empty_like(u)
        du = torch.empty_like(u)
        vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device=dev)
        buf = torch.empty((samples, L.n_dof), dtype=torch.float64, device=dev)
        for k in range(newton_steps):
            if pairs is not None and used >= pairs:
                break
            ctx.form_jacobian_fd(u, res, vals)
            rn = float(torch.linalg.vector_norm(res))
            if rn <= 1e-10:
                break
            # the samples come from the solver the correction is trained for:
            # GMRES with the base preconditioner (block-ILU(0) on the tiles)
            ctx.ilu_tile = ilu_tile
            ns, its, rr = ctx.krylov_samples(vals, res, du, buf, every=every)
            if pairs is not None:
                ns = min(ns, pairs - used)
            used += ns
            t0 = time.time()
            rep = ctx.lpc_train(vals, buf, ns, steps=steps, batch=batch, random=random, sweeps=sweeps, lr=lr,
                                seed=seed * 7919 + k)
            rec = dict(seed=seed, re=re, newton_step=k, r=rn, samples=ns, pairs_used=used, gmres_its=its,
                       loss_first=rep.loss_first, loss_last=rep.loss_last, train_s=time.time() - t0)
            out.append(rec)
            if log:
                log(rec)
            u -= du
        ctx.lpc_attach(None)
        del wl
    return out


def calibrate(model, instance, n=256, samples=167, every=5, sweeps=0, ilu_tile=0, newton_steps=2, device=0):
    """held-out check of a trained model: on the Krylov residuals of a fresh
    instance's first Newton steps, the share g in [0, 1] of the correction,
    z = (I + g C) y, that minimises the training loss (quadratic in g: the
    loss is S_aa - 2 g S_ab + g^2 S_bb); the output layer (W3, b3), on which
    C depends linearly, is scaled by g. Returns a record of g and the loss at
    g = 0 (the base preconditioner), g = 1 and the chosen g."""
    import torch
    dev = torch.device("cuda", device)
    wl = make_instance(*instance, n, device)
    ctx = wl.ctx
    L = ctx.layout
    bs = L.block_size
    u = torch.from_numpy(wl.u0).to(dev)
    res, du = torch.empty_like(u), torch.empty_like(u)
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device=dev)
    buf = torch.empty((samples, L.n_dof), dtype=torch.float64, device=dev)
    s_ab = s_bb = s_aa = 0.0
    for k in range(newton_steps):
        ctx.form_jacobian_fd(u, res, vals)
        if float(torch.linalg.vector_norm(res)) <= 1e-10:
            break
        ctx.ilu_tile = ilu_tile
        ns, _, _ = ctx.krylov_samples(vals, res, du, buf, every=every)
        ctx.lpc_attach(model)
        ab, bb, aa = ctx.lpc_calibrate(vals, buf, ns, sweeps)
        ctx.lpc_attach(None)
        s_ab, s_bb, s_aa = s_ab + ab, s_bb + bb, s_aa + aa
        u -= du
    g = min(max(s_ab / s_bb, 0.0), 1.0) if s_bb > 0 else 0.0
    p = model.get_params()
    D, H = bs * bs, model.hidden
    o_w3 = H * D + H + H * 2 * H + H
    p[o_w3:] *= g
    model.set_params(p)
    del wl
    return dict(instance=list(instance), g=g, loss_base=s_aa, loss_full=s_aa - 2 * s_ab + s_bb,
                loss_scaled=s_aa - 2 * g * s_ab + g * g * s_bb)


def correction_is_zero(model):
    """whether the model's output layer (W3, b3) is all zero: its correction
    C is then 0 and preconditioner 5 applies its base alone"""
    D, H = model.bs * model.bs, model.hidden
    o_w3 = H * D + H + H * 2 * H + H
    return not np.any(model.get_params()[o_w3:])


def select_scale(model, instance, n=256, sweeps=0, ilu_tile=0, candidates=(0.0, 0.25, 0.5, 1.0), device=0):
    """the share g of the correction chosen by what it is for: the learned,
    mixed-precision Newton solve of a held-out instance to |r| <= 1e-10 is
    run with the output layer scaled by each candidate g, and the g with the
    fewest GMRES iterations is kept (ties: the smaller g; g = 0 is the base
    preconditioner itself). The output layer of `model` is left scaled by it.
    Returns a record of the iterations per candidate and the choice."""
    p0 = model.get_params()
    D, H = model.bs * model.bs, model.hidden
    o_w3 = H * D + H + H * 2 * H + H
    wl = make_instance(*instance, n, device)
    its = {}
    for g in candidates:
        p = p0.copy()
        p[o_w3:] *= g
        model.set_params(p)
        rec, _ = solve(wl, model, 5, 1, sweeps, device, ilu_tile)
        its[g] = (rec["gmres_its"] + (10**9 if not rec["converged"] else 0), rec["s"], rec["pc_fallbacks"])
    best = min(candidates, key=lambda g: (its[g][0], g))
    p = p0.copy()
    p[o_w3:] *= best
    model.set_params(p)
    del wl
    return dict(instance=list(instance), g=best,
                candidates={str(g): dict(gmres_its=v[0], s=v[1], pc_fallbacks=v[2]) for g, v in its.items()})


def solve(wl, model=None, preconditioner=2, precision=0, sweeps=1, device=0, ilu_tile=0, matrix_free=0,
          cgs_refine=0):
    """one Newton solve of an instance to |r| <= 1e-10 (GMRES(30) with
    PETSc's default orthogonalisation, one classical Gram-Schmidt pass per
    step unless cgs_refine = 1; Wolfe line search), timed with CUDA events;
    matrix_free = 1: the GMRES operator is the residual's directional
    difference (the assembled Jacobian then only preconditions); returns
    (report dict, final state)"""
    import torch
    dev = torch.device("cuda", device)
    opt = default_newton_options()
    opt.preconditioner = preconditioner
    opt.precision = precision
    opt.pc_sweeps = sweeps
    opt.ilu_tile = ilu_tile
    opt.matrix_free = matrix_free
    opt.gmres_cgs_refine = cgs_refine
    opt.gmres_max_it = 20000
    if model is not None:
        wl.ctx.lpc_attach(model)
    u = torch.from_numpy(wl.u0).to(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    rep = wl.ctx.newton_solve(u, opt)
    e1.record()
    torch.cuda.synchronize(dev)
    if model is not None:
        wl.ctx.lpc_attach(None)
    return dict(s=e0.elapsed_time(e1) * 1e-3, ilu_tile=ilu_tile, matrix_free=matrix_free, cgs_refine=cgs_refine,
                newton_its=rep.iterations,
                gmres_its=rep.linear_iterations_total,
                gmres_its_per_step=list(rep.linear_iterations[:rep.iterations]), r_final=rep.r_final,
                converged=bool(rep.converged), pc_fallbacks=rep.pc_fallbacks), u.cpu().numpy()


def evaluate(model, eval_instances, n=256, sweeps=0, device=0, log=None, ilu_tile=0):
    """plain all-FP64 block-ILU(0) against learned + mixed precision (and the
    untrained base preconditioner, mixed, as ablation) on fresh instances"""
    out = []
    for (seed, re) in eval_instances:
        wl = make_instance(seed, re, n, device)
        plain, u_plain = solve(wl, None, 2, 0, device=device)
        learned, u_l = solve(wl, model, 5, 1, sweeps, device, ilu_tile)
        ablation, u_a = solve(wl, None, 4 if sweeps > 0 else 2, 1, sweeps, device, ilu_tile)
        scale = max(np.linalg.norm(u_plain), 1e-300)
        rec = dict(seed=seed, re=re, plain_fp64_ilu0=plain, learned_mixed=learned, untrained_base_mixed=ablation,
                   learned_vs_plain_state_l2=float(np.linalg.norm(u_l - u_plain) / scale),
                   speedup_learned_mixed_vs_plain_fp64=plain["s"] / learned["s"],
                   speedup_untrained_base_mixed_vs_plain_fp64=plain["s"] / ablation["s"])
        out.append(rec)
        if log:
            log(rec)
        del wl
    return out


def new_model(device=0, seed=0, hidden=256):
    return LearnedPreconditioner(BLOCK_SIZE, hidden, device, seed)


# the training recipe of the shipped model (data/learned_pc_ns_p2.npz): 2,000
# Jacobian / residual pairs from the plain solver on seeded instances (Re
# uniform in [50, 500]), the correction trained on top of block-ILU(0) on
# 32 x 32 element tiles with exact triangular solves (pc_sweeps = 0), then
# scaled on a held-out instance: by the training loss (calibrate), then by the
# GMRES iterations of its Newton solve (select_scale)
RECIPE = dict(model_seed=1, train_instances=(8, 11), pairs=2000, samples=167, every=5, steps=120, batch=4, random=2,
              sweeps=0, ilu_tile=8, lr=1e-3, holdout=(1, 5))
EVAL_INSTANCES = (3, 99)


def main(argv=None):
    """python -m iceicle_b200.learned_pc train OUT.npz | evaluate MODEL.npz"""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("path")
    ap.add_argument("--n", type=int, default=256, help="quadrilaterals per direction")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        r = RECIPE
        m = new_model(seed=r["model_seed"])
        train(m, instances(*r["train_instances"]), n=a.n, samples=r["samples"], every=r["every"], steps=r["steps"],
              batch=r["batch"], random=r["random"], sweeps=r["sweeps"], lr=r["lr"], pairs=r["pairs"],
              ilu_tile=r["ilu_tile"], log=lambda x: print(json.dumps(x), flush=True))
        hold = instances(*r["holdout"])[0]
        rec = calibrate(m, hold, n=a.n, samples=r["samples"], every=r["every"], sweeps=r["sweeps"],
                        ilu_tile=r["ilu_tile"])
        print(json.dumps({"calibration": rec}), flush=True)
        rec = select_scale(m, hold, n=a.n, sweeps=r["sweeps"], ilu_tile=r["ilu_tile"])
        print(json.dumps({"selection": rec}), flush=True)
        m.save(a.path, sweeps=r["sweeps"], ilu_tile=r["ilu_tile"])
    else:
        m = LearnedPreconditioner.load(a.path)
        evaluate(m, instances(*EVAL_INSTANCES), n=a.n, sweeps=m.sweeps, ilu_tile=m.ilu_tile or 0,
                 log=lambda x: print(json.dumps(x), flush=True))


if __name__ == "__main__":
    main()
