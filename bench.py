"""Benchmark of the DG residual hot path: DOF-residual evaluations per second
on the 2D compressible Navier-Stokes manufactured-solution workload
(128 x 128 quads, p = 3, geometry order 2 with seeded curved-node
perturbation, 5x5 / 5-point Gauss-Legendre, Van Leer + interior penalty, FP64).

One step = one full residual evaluation R(u) of the whole mesh
(form_residual, src/solvers/include/iceicle/form_residual.hpp:56-268).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed.run with the mesh partitioned into
element-row strips (iceicle_b200.partition; weak scaling: every rank owns a
128 x 128 strip of a 128 x 128 N mesh). A step is then the halo exchange of
one coefficient row per neighbour over NCCL plus the rank's residual. The
timed region is bracketed by a barrier and synchronisations and the time is
the maximum over ranks. --impl reference times the reference's own CPU
implementation (its headers compiled as oracle/_ref) on the host cores.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload="ns_mms_residual", pde="navier_stokes", mesh="128x128 quads", p=3, geometry_order=2,
                quadrature="5x5 volume / 5 face Gauss-Legendre", conv_flux="van_leer", diffusive="interior_penalty",
                node_perturbation="smooth seeded, 0.05 h", n_dof=1048576,
                l2="inputs < L2; L2 flushed (256 MiB write) between timed steps")
METRIC = "DOF-residual evals/s"
NX = NY = 128


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-newton", action="store_true", help="skip the secondary Newton solve timings")
    ap.add_argument("--spmv", type=int, default=0, metavar="N",
                    help="only time the FP64 BSR SpMV of the N x N p = 2 Navier-Stokes Jacobian (36 x 36 blocks) "
                         "and print one JSON line")
    ap.add_argument("--ilu", type=int, default=0, metavar="N",
                    help="only time the block-ILU(0) apply (data-flow and row-pipelined, FP64 and FP32 factors) "
                         "of the N x N p = 2 Navier-Stokes Jacobian and print one JSON line")
    ap.add_argument("--factor", action="store_true",
                    help="only time the block-ILU(0) factorisation (Burgers 32 x 32 p = 2, NS 128 x 128 p = 3, "
                         "NS 256 x 256 p = 2) and print one JSON line")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-preconditioner Newton comparison (256 x 256 Navier-Stokes, p = 2)")
    ap.add_argument("--batched", type=int, default=512, metavar="N",
                    help="secondary timing of N seeded uneven advection-diffusion problems, batched vs one at a "
                         "time (0: skip; the full problem set is 512)")
    ap.add_argument("--batched-sample", type=int, default=16, metavar="K",
                    help="problems of the set also solved one at a time for the batched ratio")
    ap.add_argument("--batched-fp32q", action="store_true",
                    help="also time the problem set with FP32 flux quadrature (precision 2)")
    ap.add_argument("--learned-seeds", type=int, default=1, metavar="K",
                    help="fresh instances of the learned-preconditioner comparison (256 x 256 Navier-Stokes)")
    ap.add_argument("--no-lm", action="store_true", help="skip the MDG-ICE (64 x 64) LM timing")
    ap.add_argument("--gemm", default="", metavar="M,N,K",
                    help="only time the tcgen05 BF16 GEMM out = A B^T (A [M, K], B [N, K], FP32 out) and print "
                         "one JSON line")
    ap.add_argument("--jacobian", type=int, default=0, metavar="N",
                    help="only time the FD Jacobian (FP64 and FP32 flux quadrature) of the N x N p = 3 "
                         "Navier-Stokes manufactured solution and print one JSON line")
    ap.add_argument("--solve", type=int, default=-1, metavar="TILE",
                    help="only run one Newton solve of the first evaluation instance of the 256 x 256 p = 2 "
                         "Navier-Stokes problem (autotuned shapes) with block-ILU(0) on TILE x TILE element "
                         "tiles (0: the whole grid) and print one JSON line")
    ap.add_argument("--solve-precision", type=int, default=1, metavar="P",
                    help="Newton precision of --solve (0 FP64, 1 mixed, 2 FP32 flux quadrature)")
    ap.add_argument("--solve-matrix-free", action="store_true",
                    help="--solve with the matrix-free GMRES operator (residual differences)")
    ap.add_argument("--no-tune", action="store_true",
                    help="time the compiled default launch shapes instead of the autotuned ones")
    ap.add_argument("--tile", default="", metavar="K=V,...",
                    help="time the residual with these launch shapes instead of autotuning them, e.g. "
                         "face_minb=4,vol_threads=128,vol_minb=8 (for profiling the shapes a plain run chose)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------ CPU baseline
def _ref_worker(args):
    """time the reference's form_residual on the full workload in one process:
    the same mesh nodes and initial state as the GPU arm (manufactured state
    at the basis nodes with the seeded 1e-3 noise), built from the oracle's
    own workload callbacks so that this process maps no product library.
    Returns (unknowns, seconds per residual, loaded product libraries)."""
    nrep, _ = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bindings as ob
    from specs import NS, Spec
    spec = Spec(pde=NS, nx=NX, ny=NY, p=3, g=2, ip=True, source=True, perturb=0.05, seed=4321)
    pb = spec.oracle_problem()
    c = spec.coords()
    u = spec.mms_state(c, seed=4321, noise=1e-3)
    s = C.c_double()
    rc = ob.ref().fn("time_form_residual")(C.byref(pb), c.ctypes.data_as(C.c_void_p),
                                           u.ctypes.data_as(C.c_void_p), nrep, C.byref(s))
    assert rc == 0
    return spec.N, s.value, _mapped_product_libs()


def _mapped_product_libs():
    """product shared objects mapped into this process (the reference arm must map none)"""
    try:
        with open("/proc/self/maps") as f:
            return sorted({ln.split()[-1] for ln in f if "libiceicle_b200" in ln})
    except OSError:
        return []


def cpu_reference(nrep, procs):
    """aggregate throughput of `procs` concurrent single-threaded reference
    processes (the reference is serial per MPI rank), each evaluating the full
    workload `nrep` times"""
    import multiprocessing as mp
    if procs == 1:
        res = [_ref_worker((nrep, 0))]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            res = pool.map(_ref_worker, [(nrep, i) for i in range(procs)])
    value = sum(r[0] / r[1] for r in res)
    return value, res


def run_reference(a):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bindings as ob
    if not ob.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref not present"}))
        return
    procs = os.cpu_count() or 1
    t0 = time.time()
    # each process: one untimed warm-up evaluation, then `steps` timed ones
    value, res = cpu_reference(a.steps, procs)
    wall = time.time() - t0
    mapped = sorted({m for r in res for m in r[2]})
    assert not mapped, f"reference arm mapped product libraries: {mapped}"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": 0,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * np.mean([r[1] for r in res]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded manufactured solution)", "config": WORKLOAD, "parallelism": "host processes",
        "cpu_baseline": {"value": value, "unit": "DOF/s", "cores": procs, "kind": "reference",
                         "sample": f"{procs} concurrent processes x full 128x128 p3 residual (reference headers, -O3)"},
        "e2e": {"value": value, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall, "product_libs_mapped": mapped,
    }
    print(json.dumps(line))


# ------------------------------------------------------------- GPU arm
class ClockSampler:
    def __init__(self, index):
        self.proc = None
        import tempfile
        try:
            self.f = tempfile.NamedTemporaryFile("w", prefix="icx_clocks_", suffix=".csv", delete=False)
            self.out = self.f.name
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        rows = []
        with open(self.out) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 7:
                    rows.append(parts)
        os.unlink(self.out)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def residual_work(wl):
    """algorithmic bytes and FP64 flops per launch of the two residual kernels.
    Bytes: every array the kernel must touch, once (u, res, geometry, source,
    boundary data, the face fluxes passed between the kernels). Flops: the
    sum-factorised contractions as implemented (2 per multiply-add) plus
    160 per Navier-Stokes physical flux and 420 per numerical flux (Van Leer
    splitting of both states + viscous flux), counted once per point."""
    L = wl.ctx.layout
    E, nb, neq, nqv, nqf, F = L.n_elem, L.nbasis, L.neq, L.nq_vol, L.nq_face, L.n_faces
    N = L.n_dof
    n1 = int(round(nb ** 0.5))
    q1 = nqf
    bytes_vol = 8 * (2 * N + E * nqv * (5 + neq) + F * nqf * neq)
    bytes_face = 8 * (N + F * nqf * 12 + F * nqf * neq)
    fma_vol = (n1 * q1 * neq * 2 * n1 + nqv * neq * 3 * n1 + nqv * neq * 10 + q1 * n1 * neq * 3 * q1
               + 4 * n1 * nqf * neq + nb * neq * (2 * q1 + 4))
    flops_vol = E * (2 * fma_vol + nqv * 160)
    fma_face = F * (2 * neq * n1 * 2 * n1 + nqf * 2 * neq * (3 * n1 + 4))
    flops_face = 2 * fma_face + F * nqf * 420
    return dict(vol=(bytes_vol, flops_vol), face=(bytes_face, flops_face))


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the two
# residual kernels on this workload in the tuned shapes (the default shapes
# read the same: 43.45 MB and 25.59 MB), from one ncu capture of
#   ncu --section SpeedOfLight --section MemoryWorkloadAnalysis --section Occupancy \
#       --section WarpStateStats --section LaunchStats \
#       --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none \
#       -k "regex:vol_lift|face_flux" -s 4 -c 2 python bench.py --steps 2 --warmup 3 \
#       --no-newton --no-cpu-baseline --batched 0 --no-learned \
#       --tile face_minb=4,vol_threads=128,vol_minb=8
NCU_DRAM_BYTES = {"vol": 43.45e6 + 0.57e6, "face": 25.42e6 + 0.0003e6}


def batched_bench(torch, dev, n_problems, sample=16, fp32_quadrature=False):
    """Newton solves to |r| <= 1e-10 per problem (Wolfe line search, GMRES(30)
    + block-ILU(0)) of the seeded uneven advection-diffusion problems (meshes
    8x8 to 96x96, orders 1-4, viscosity log-uniform in [1e-4, 1e-1], advection
    angle uniform): all of them as one ProblemSet (each problem its own Newton
    solve; every kernel launched once per basis order for all problems; each
    Arnoldi step of the set one CUDA graph), in FP64 and with FP32 flux
    quadrature (precision 2), against the problems solved one context at a
    time. One at a time runs on a seeded sample of `sample` problems (all of
    them would take minutes); the ratio compares it with the set of the same
    sample. Every timing is the second of two runs (the first does the
    one-time setup: buffers, graph capture); CUDA events around each solve;
    contexts are built before the timed region."""
    import iceicle_b200 as ib
    import iceicle_b200.workloads as w
    specs = w.batched_problem_specs(n_problems)
    parts, u0 = [], []
    for sp in specs:
        c, u = w.advection_diffusion_problem(sp, dev.index)
        parts.append(c)
        u0.append(u)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize(dev)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) * 1e-3, out

    def set_solve(ps, prec):
        opt = ib.default_newton_options()
        opt.precision = prec
        holder = {}

        def run():
            u = torch.from_numpy(ps.gather([u0[k] for k in ps.members])).to(dev)
            holder["u"] = u
            return ps.newton_solve(u, opt)
        t, (reps, stats) = timed(run)
        return t, holder["u"].cpu().numpy(), reps, stats

    ps = ib.ProblemSet(parts, dev.index)
    ps.members = list(range(n_problems))
    t_all, u_all, reps, stats = set_solve(ps, 0)
    t_q32, u_q32, reps32 = (set_solve(ps, 2)[:3]) if fp32_quadrature else (None, u_all, reps)
    rng = np.random.default_rng(5)
    pick = sorted(rng.choice(n_problems, size=min(sample, n_problems), replace=False).tolist())
    sub = ib.ProblemSet([parts[k] for k in pick], dev.index)
    sub.members = pick
    t_sub, u_sub, _, _ = set_solve(sub, 0)
    opt = ib.default_newton_options()
    t_seq, worst = 0.0, 0.0
    for i, k in enumerate(pick):
        holder = {}

        def run():
            uk = torch.from_numpy(u0[k].copy()).to(dev)
            holder["u"] = uk
            return parts[k].newton_solve(uk, opt)
        t, _ = timed(run)
        t_seq += t
        a, b = holder["u"].cpu().numpy(), sub.part(u_sub, i)
        worst = max(worst, float(np.linalg.norm(a - b) / max(np.linalg.norm(a), 1e-300)))
    q32 = max(float(np.linalg.norm(ps.part(u_all, k) - ps.part(u_q32, k)) /
                    max(np.linalg.norm(ps.part(u_all, k)), 1e-300)) for k in range(n_problems)) \
        if fp32_quadrature else None
    n_dof = ps.offsets[-1]
    out = {"problems": n_problems, "n_dof": int(n_dof), "orders": stats.orders,
           "set_fp64_s": t_all, "set_fp32_quadrature_s": t_q32,
           "converged": int(sum(r.converged for r in reps)), "converged_fp32_quadrature": int(sum(r.converged for r in reps32)) if fp32_quadrature else None,
           "newton_rounds": stats.newton_rounds, "arnoldi_steps": stats.arnoldi_steps,
           "arnoldi_graph_launches": stats.graph_launches, "line_search_rounds": stats.line_search_rounds,
           "max_newton_its": max(r.iterations for r in reps),
           "fp32_quadrature_vs_fp64_state_l2_max": q32,
           "sample": {"problems": len(pick), "set_s": t_sub, "one_at_a_time_s": t_seq,
                      "speedup": t_seq / t_sub if t_sub > 0 else None, "max_state_rel_diff": worst}}
    sub.close()
    ps.close()
    return out


def roe_residual_bench(torch, dev, flush, tune=True, steps=20):
    """the residual workload with the Roe convective flux the configuration
    names (the headline line keeps Van Leer, the flux the reference has, so
    that both arms time the same discretization): device time per residual
    with L2 flushed between steps"""
    import iceicle_b200 as ib
    from iceicle_b200.workloads import ns_mms_config
    wl = ns_mms_config(nx=NX, ny=NY, p=3, geo_order=2, device=dev.index, conv_flux=ib.FLUX_ROE)
    u = torch.from_numpy(wl.u0).to(dev)
    res = torch.empty_like(u)
    if tune:
        wl.ctx.autotune(u, ib.TUNE_RESIDUAL)
    for _ in range(3):
        wl.ctx.form_residual(u, res)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize(dev)
    for e0, e1 in ev:
        flush.zero_()
        e0.record()
        wl.ctx.form_residual(u, res)
        e1.record()
    torch.cuda.synchronize(dev)
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps
    n = wl.ctx.layout.n_dof
    del wl
    return {"conv_flux": "roe", "ms": ms, "dof_per_s": n / (ms * 1e-3)}


def jacobian_work(L):
    """algorithmic bytes (BSR values written once, u read) and an FP64 flop
    count of one FD Jacobian as the element kernel computes it: per element
    and perturbed DOF, the four faces' point states and numerical fluxes
    (420 flops per Navier-Stokes face flux, 28 per state update) and their
    contraction into the two blocks a face column touches; per element the
    flux-level volume FD (1 + 3 neq physical fluxes of 160 flops per point)
    and its contraction into the diagonal block (12 flops per entry and point)"""
    E, nb, neq, nqv, nqf = L.n_elem, L.nbasis, L.neq, L.nq_vol, L.nq_face
    bs = nb * neq
    face = bs * 4 * nqf * (28 + 420) + 2 * nb * neq * bs * nqf * 4 * 2
    vol = nqv * (1 + 3 * neq) * 160 + bs * bs * nqv * 12
    bytes_ = L.nnz_blocks * bs * bs * 8 + L.n_dof * 8
    return bytes_, E * (face + vol)


def jacobian_bench(torch, dev, wl, hbm_gbs, cpu=True):
    """FD Jacobian (form_petsc_jacobian_fd) of the residual workload into BSR:
    mean device time of 5 launches after 2 untimed ones (CUDA events), the
    BSR bytes it writes, GB/s against the measured HBM peak, FP64 flops; and
    the reference's own form_petsc_jacobian_fd on one host core, timed on a
    32 x 32 sample of the same discretization and scaled by the element count
    (its cost is linear in the elements)"""
    L = wl.ctx.layout
    bs = L.block_size
    u = torch.from_numpy(wl.u0).to(dev)
    res = torch.empty_like(u)
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device=dev)
    for _ in range(2):
        wl.ctx.form_jacobian_fd(u, res, vals)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(5):
        wl.ctx.form_jacobian_fd(u, res, vals)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / 5
    nbytes, flops = jacobian_work(L)
    out = {"workload": "ns_mms 128x128 p3 (the residual workload)", "ms": ms, "bsr_bytes": L.nnz_blocks * bs * bs * 8,
           "algorithmic_bytes": nbytes, "GBs": nbytes / ms / 1e6, "frac_of_hbm": nbytes / ms / 1e6 / hbm_gbs,
           "fp64_flops": flops, "fp64_tflops": flops / ms / 1e9}
    del vals
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_bindings as ob
        if ob.ref_available():
            from specs import NS, Spec
            n = 32
            spec = Spec(pde=NS, nx=n, ny=n, p=3, g=2, ip=True, source=True, perturb=0.05, seed=4321)
            pb = spec.oracle_problem()
            c = spec.coords()
            us = spec.mms_state(c)
            rp, ci = ob.bsr_pattern(pb)
            hv = np.zeros(len(ci) * bs * bs)
            sec = C.c_double()
            rc = ob.ref().fn("time_jacobian_fd")(C.byref(pb), ob._ptr(c), ob._ptr(us), ob._ptr(rp), ob._ptr(ci),
                                                 ob._ptr(hv), 1, C.byref(sec))
            if rc == 0:
                scale = L.n_elem / (n * n)
                out["cpu_reference"] = {"ms": sec.value * 1e3 * scale, "cores": 1,
                                        "sample": f"{n}x{n} p3 (same physics), 1 call after a warm-up, x{scale:g} "
                                                  "elements (linear in the element count)"}
                out["speedup_vs_cpu_reference"] = sec.value * 1e3 * scale / ms
    return out


def lm_bench(torch, dev, kmax=1, maxit=300, orders=(1,)):
    """MDG-ICE (CorriganLM with the explicitly formed, ILU(0)-preconditioned
    subproblem): 64 x 64 quads, p = 1 and p = 2, oblique inviscid-Burgers
    shock on a jittered grid, all interior traces selected; wall time of
    `kmax` LM iterations (CUDA events around the solve) with at most `maxit`
    GMRES(60) iterations per subproblem, the residual history, the linear
    iterations and the worst relative residual a subproblem solve ended with
    (the reference's GMRES + ILU(0) does not reach small tolerances on this
    system at this size)"""
    import iceicle_b200 as ib
    from iceicle_b200.workloads import mdg_ice_config
    out = {}
    for p in orders:
        wl, traces, x0 = mdg_ice_config(n=64, p=p, device=dev.index)
        o = ib.default_lm_options()
        o.kmax, o.explicit_subproblem, o.gmres_rtol, o.gmres_max_it, o.gmres_restart = kmax, 1, 1e-8, maxit, 60
        u = torch.from_numpy(wl.u0.copy()).to(dev)
        x = x0.copy()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record()
        rep = ib.lm_solve(wl.ctx, u, x, o)
        e1.record()
        torch.cuda.synchronize(dev)
        out[f"mdg_ice_64x64_p{p}"] = {
            "s": e0.elapsed_time(e1) * 1e-3, "iterations": rep.iterations, "rejections": rep.rejections,
            "gmres_its": rep.linear_iterations_total, "n_geo": len(x0),
            "subproblem_relres_max": rep.linear_relres_max,
            "residual_history": list(rep.residual_history[:rep.iterations + 1])}
        del wl
    return out


def newton_bench(torch, dev, tune=True):
    """Newton solve time to |r| <= 1e-10 (FP64 residual; GMRES with PETSc's
    default orthogonalisation, one classical Gram-Schmidt pass), all-FP64 vs mixed
    precision (FP32 Jacobian and preconditioner copies) and FP32 flux
    quadrature (the Jacobian itself formed in FP32): 32 x 32 viscous
    Burgers p=2 and the 128 x 128 Navier-Stokes manufactured solution p=3,
    both with GMRES(30) + block-ILU(0) and the Wolfe line search. Timed with
    CUDA events around the whole solve (it synchronises internally). With
    `tune`, the residual and ILU launch shapes are autotuned at the initial
    state first (outside the timed solves)."""
    import iceicle_b200 as ib
    from iceicle_b200.workloads import burgers_config, ns_mms_config
    out = {}
    for name, make in (("burgers_32x32_p2", lambda: burgers_config(device=dev.index)),
                       ("ns_mms_128x128_p3", lambda: ns_mms_config(nx=NX, ny=NY, p=3, geo_order=2,
                                                                    device=dev.index))):
        wl = make()
        rows = {}
        if tune:
            t = wl.ctx.autotune(torch.from_numpy(wl.u0).to(dev),
                                ib.TUNE_RESIDUAL | ib.TUNE_ILU | ib.TUNE_ILU_FP32)
            rows["autotune"] = {"chosen": t["chosen"], "from_cache": t["from_cache"],
                                "ilu_ms_default": t["ilu_ms_default"], "ilu_ms_tuned": t["ilu_ms_tuned"]}
        states = {}
        tile = 8 if name.startswith("burgers") else 16
        for label, prec, t, mf in (("fp64", 0, 0, 0), ("mixed", 1, 0, 0), ("mixed_tiled", 1, tile, 0),
                                   ("quad32_tiled", 2, tile, 0), ("bf16_tiled_matrix_free", 3, tile, 1)):
            if tune and t and "autotune_tiled" not in rows:
                # the apply's launch shapes for the tiled pattern
                wl.ctx.ilu_tile = t
                t2 = wl.ctx.autotune(torch.from_numpy(wl.u0).to(dev), ib.TUNE_ILU | ib.TUNE_ILU_FP32)
                rows["autotune_tiled"] = {"chosen": t2["chosen"], "ilu_ms_default": t2["ilu_ms_default"],
                                          "ilu_ms_tuned": t2["ilu_ms_tuned"]}
            opt = ib.default_newton_options()
            opt.precision = prec
            opt.ilu_tile = t
            opt.matrix_free = mf
            opt.gmres_cgs_refine = 0  # PETSc's default GMRES orthogonalisation (one Gram-Schmidt pass)
            u = torch.from_numpy(wl.u0).to(dev)
            if name.startswith("burgers"):
                wl.ctx.newton_solve(torch.from_numpy(wl.u0).to(dev), opt)  # warm-up (one-time setup)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record()
            rep = wl.ctx.newton_solve(u, opt)
            e1.record()
            torch.cuda.synchronize(dev)
            states[label] = u.cpu().numpy()
            rows[label] = {"s": e0.elapsed_time(e1) * 1e-3, "ilu_tile": t, "matrix_free": mf, "newton_its": rep.iterations,
                           "gmres_its": rep.linear_iterations_total, "r_final": rep.r_final,
                           "converged": bool(rep.converged)}
        a = states["fp64"]
        for label in ("mixed", "mixed_tiled", "quad32_tiled", "bf16_tiled_matrix_free"):
            rows[f"{label}_vs_fp64_state_l2"] = float(np.linalg.norm(a - states[label]) /
                                                      max(np.linalg.norm(wl.u0), 1e-300))
            rows[f"speedup_{label}_vs_fp64"] = rows["fp64"]["s"] / rows[label]["s"]
        out[name] = rows
        del wl
    return out


def spmv_bench(n):
    """FP64 BSR SpMV of the FD Jacobian of the n x n p = 2 Navier-Stokes
    manufactured solution (36 x 36 blocks): 3 untimed, then 20 timed launches
    between CUDA events; inputs larger than L2 from n = 96 on"""
    import torch
    from iceicle_b200.workloads import ns_mms_config
    dev = torch.device("cuda", 0)
    wl = ns_mms_config(nx=n, ny=n, p=2, geo_order=2, mu=0.01)
    ctx, L = wl.ctx, wl.ctx.layout
    bs = L.block_size
    u = torch.from_numpy(wl.u0).to(dev)
    res = torch.empty_like(u)
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device=dev)
    ctx.form_jacobian_fd(u, res, vals)
    x = torch.randn(L.n_dof, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
    y = torch.empty_like(x)
    for _ in range(3):
        ctx.bsr_spmv(vals, x, y)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(20):
        ctx.bsr_spmv(vals, x, y)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / 20
    nbytes = L.nnz_blocks * bs * bs * 8 + L.nnz_blocks * 4 + (L.n_elem + 1) * 4 + 2 * L.n_dof * 8
    print(json.dumps({"spmv": f"ns_mms_{n}x{n}_p2", "block": bs, "ms": ms, "algorithmic_bytes": nbytes,
                      "GBs": nbytes / ms / 1e6}))


def ilu_bench(n):
    """block-ILU(0) apply of the FD Jacobian of the n x n p = 2 Navier-Stokes
    manufactured solution: mean of 20 applies after 3 untimed ones, per
    schedule and precision (CUDA events inside icx_ilu_apply). The first
    ilu_apply_flow_kernel launches are the FP64 sentinel-schedule ones."""
    import torch
    from iceicle_b200.workloads import ns_mms_config
    dev = torch.device("cuda", 0)
    wl = ns_mms_config(nx=n, ny=n, p=2, geo_order=2, mu=0.01)
    ctx, L = wl.ctx, wl.ctx.layout
    bs = L.block_size
    u = torch.from_numpy(wl.u0).to(dev)
    res = torch.empty_like(u)
    vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device=dev)
    ctx.form_jacobian_fd(u, res, vals)
    x = torch.randn(L.n_dof, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
    y = torch.empty_like(x)
    out = {"ilu": f"ns_mms_{n}x{n}_p2", "block": bs, "levels_per_sweep": 2 * n - 1}
    # the data-flow apply (default rows per task and CTAs per SM) on its two
    # schedules, then the row-pipelined apply
    for sched, sn in ((2, "sentinel"), (1, "counters")):
        ctx.tile = {"ilu_sched": [sched, sched]}
        for prec, pn in ((0, "fp64"), (1, "fp32")):
            ctx.ilu_apply(vals, x, y, prec, 1, 3)
            out[f"data_flow_{sn}_{pn}_ms"] = ctx.ilu_apply(vals, x, y, prec, 1, 20)
    ctx.tile = {}
    for prec, pn in ((0, "fp64"), (1, "fp32")):
        ctx.ilu_apply(vals, x, y, prec, 2, 3)
        out[f"rows_{pn}_ms"] = ctx.ilu_apply(vals, x, y, prec, 2, 20)
    # the data-flow apply with the autotuned schedule, rows per task and CTAs per SM
    import iceicle_b200 as ib
    t = ctx.autotune(u, ib.TUNE_ILU | ib.TUNE_ILU_FP32)
    out["tuned_tile"] = {k: t["chosen"][k] for k in ("ilu_rows", "ilu_ctas", "ilu_sched")}
    for prec, pn in ((0, "fp64"), (1, "fp32")):
        ctx.ilu_apply(vals, x, y, prec, 1, 3)
        out[f"data_flow_tuned_{pn}_ms"] = ctx.ilu_apply(vals, x, y, prec, 1, 20)
    # block-ILU(0) on element tiles (block-Jacobi over the tiles): fewer dependent levels, dropped couplings;
    # the per-tile apply (one CTA per tile, the default) and the data-flow apply on the tiled factors
    for tile in (8, 16, 32, 64):
        ctx.ilu_tile = tile
        # per-tile applies: one lane per row, matrix rows staged in shared memory or in registers,
        # with 512 / 256 / 128 threads per CTA (k = 1 / 2 / 3; 0 the default); the data-flow apply
        shapes = ([(5, k, f"rowpar_k{k}") for k in (0, 1, 2, 3)] + [(4, k, f"staged_k{k}") for k in (0, 1, 3)] +
                  [(3, 0, "tiles"), (2, 0, "data_flow")])
        for sched, k, sn in shapes:
            ctx.tile = {"ilu_sched": [sched, sched], "ilu_ctas": [k, k]}
            # BF16 factors (FP32 arithmetic) only in the one-lane-per-row form
            for prec, pn in ((0, "fp64"), (1, "fp32")) + (((2, "bf16"),) if sched == 5 else ()):
                ctx.ilu_apply(vals, x, y, prec, 0, 3)
                out[f"tiled{tile}_{sn}_{pn}_ms"] = ctx.ilu_apply(vals, x, y, prec, 0, 20)
    ctx.tile = {}
    ctx.ilu_tile = 0
    # bytes one apply must read: the off-diagonal factor blocks and the E diagonal inverses (one matrix's worth)
    out["factor_bytes_fp64"] = L.nnz_blocks * bs * bs * 8
    print(json.dumps(out))


def factor_bench():
    """block-ILU(0) factorisation time (one launch per anti-diagonal level plus
    the upper-block scaling): host wall time of one icx_ilu_apply with a single
    apply, minus that apply's device time, best of 3 after a warm-up. The
    first ilu_level_kernel launches are the Burgers workload's."""
    import torch
    from iceicle_b200.workloads import burgers_config, ns_mms_config
    out = {"factor": "block-ILU(0), FP64"}
    for name, make in (("burgers_32x32_p2", lambda: burgers_config()),
                       ("ns_mms_128x128_p3", lambda: ns_mms_config(nx=128, ny=128, p=3, geo_order=2)),
                       ("ns_mms_256x256_p2", lambda: ns_mms_config(nx=256, ny=256, p=2, geo_order=2, mu=0.01))):
        wl = make()
        ctx, L = wl.ctx, wl.ctx.layout
        bs = L.block_size
        u = torch.from_numpy(wl.u0).cuda()
        res = torch.empty_like(u)
        vals = torch.empty(L.nnz_blocks * bs * bs, dtype=torch.float64, device="cuda")
        ctx.form_jacobian_fd(u, res, vals)
        x = torch.randn(L.n_dof, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
        y = torch.empty_like(x)
        ctx.ilu_apply(vals, x, y, 0, 1, 2)
        ts = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ms_apply = ctx.ilu_apply(vals, x, y, 0, 1, 1)
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3 - ms_apply)
        nx = int(round((L.n_elem) ** 0.5))
        out[name] = {"block": bs, "levels": 2 * nx - 1, "factor_ms": min(ts), "us_per_level": 1e3 * min(ts) / (2 * nx - 1)}
        del wl
    print(json.dumps(out))


def learned_bench(torch, dev, tune=True, n_seeds=3):
    """Newton solve time to |r| <= 1e-10 (every row with PETSc's default
    GMRES orthogonalisation, as the reference's KSPSetFromOptions gets it) on
    fresh seeded instances of the 256 x 256 p = 2 Navier-Stokes manufactured
    solution (Re drawn from
    [50, 500]): the plain all-FP64 GMRES(30) + block-ILU(0) solve (whole grid,
    natural order) against the learned preconditioner (shipped model) in mixed
    precision on its base preconditioner (block-ILU(0) on element tiles), with
    mixed whole-grid block-ILU(0) and the untrained tiled base as references.
    CUDA events around each whole solve."""
    from iceicle_b200 import LearnedPreconditioner
    from iceicle_b200 import learned_pc as lp
    path = os.path.join(ROOT, "iceicle_b200", "data", "learned_pc_ns_p2.npz")
    if not os.path.exists(path):
        return {"unavailable": "model file iceicle_b200/data/learned_pc_ns_p2.npz absent"}
    try:
        m = LearnedPreconditioner.load(path, dev.index)
    except ValueError as exc:
        return {"unavailable": f"model file does not fit the network: {exc}"}
    sw = m.sweeps if m.sweeps is not None else 0
    tile = m.ilu_tile if m.ilu_tile is not None else 0
    # a held-out selection that kept none of the correction leaves the output
    # layer zero: preconditioner 5 is then its base (the tiled block-ILU(0))
    out = {"model": {"params": m.n_params, "pc_sweeps": sw, "ilu_tile": tile,
                     "correction_zero": bool(lp.correction_is_zero(m)),
                     "file": "iceicle_b200/data/learned_pc_ns_p2.npz"}, "instances": []}
    speed, speed_mf = [], []
    for seed, re in lp.instances(*lp.EVAL_INSTANCES)[:n_seeds]:
        wl = lp.make_instance(seed, re, 256, dev.index)
        tuned = None
        if tune:  # launch shapes for every solve below, chosen at the initial state
            import iceicle_b200 as ib
            t = wl.ctx.autotune(torch.from_numpy(wl.u0).to(dev), ib.TUNE_RESIDUAL | ib.TUNE_ILU | ib.TUNE_ILU_FP32)
            tuned = {"chosen": t["chosen"], "ilu_ms_default": t["ilu_ms_default"], "ilu_ms_tuned": t["ilu_ms_tuned"]}
        plain, u_p = lp.solve(wl, None, 2, 0, device=dev.index)
        mixed, _ = lp.solve(wl, None, 2, 1, device=dev.index)
        if tune and tile:  # the apply's launch shapes for the tiled pattern
            wl.ctx.ilu_tile = tile
            t2 = wl.ctx.autotune(torch.from_numpy(wl.u0).to(dev), ib.TUNE_ILU | ib.TUNE_ILU_FP32)
            tuned["tiled"] = {"chosen": t2["chosen"], "ilu_ms_default": t2["ilu_ms_default"],
                              "ilu_ms_tuned": t2["ilu_ms_tuned"]}
        tiled, _ = lp.solve(wl, None, 2, 1, 0, dev.index, tile)
        learned, u_l = lp.solve(wl, m, 5, 1, sw, dev.index, tile)
        # precision 3 (the tiled factors in BF16, FP32 arithmetic) with the
        # matrix-free operator (the assembled Jacobian preconditions only)
        tiled_mf, _ = lp.solve(wl, None, 2, 3, 0, dev.index, tile, matrix_free=1)
        learned_mf, u_lm = lp.solve(wl, m, 5, 3, sw, dev.index, tile, matrix_free=1)
        del wl
        rec = {"seed": seed, "re": re, "mesh": "256x256", "p": 2, "n_dof": 256 * 256 * 36,
               "plain_fp64_ilu0": plain, "mixed_ilu0": mixed, "mixed_ilu0_tiled": tiled, "learned_mixed": learned,
               "mixed_ilu0_tiled_bf16_matrix_free": tiled_mf, "learned_mixed_bf16_matrix_free": learned_mf,
               "autotune": tuned,
               "learned_vs_plain_state_l2": float(np.linalg.norm(u_l - u_p) / np.linalg.norm(u_p)),
               "learned_bf16_matrix_free_vs_plain_state_l2": float(np.linalg.norm(u_lm - u_p) / np.linalg.norm(u_p)),
               "speedup_learned_mixed_vs_plain_fp64": plain["s"] / learned["s"],
               "speedup_learned_mixed_bf16_matrix_free_vs_plain_fp64": plain["s"] / learned_mf["s"],
               "speedup_mixed_ilu0_vs_plain_fp64": plain["s"] / mixed["s"],
               "speedup_mixed_ilu0_tiled_vs_plain_fp64": plain["s"] / tiled["s"],
               "speedup_mixed_ilu0_tiled_bf16_matrix_free_vs_plain_fp64": plain["s"] / tiled_mf["s"]}
        out["instances"].append(rec)
        speed.append(rec["speedup_learned_mixed_vs_plain_fp64"])
        speed_mf.append(rec["speedup_learned_mixed_bf16_matrix_free_vs_plain_fp64"])
    out["speedup_learned_mixed_vs_plain_fp64"] = {"per_seed": speed, "min": min(speed), "mean": float(np.mean(speed)),
                                                  "target": 3.0}
    out["speedup_learned_mixed_bf16_matrix_free_vs_plain_fp64"] = {"per_seed": speed_mf, "min": min(speed_mf),
                                                                   "mean": float(np.mean(speed_mf)), "target": 3.0}
    return out


def run_ours(a):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        # the communicator is created by a collective of every rank before the
        # first point-to-point batch of the halo exchange
        dist.barrier(device_ids=[local])
    torch.cuda.set_device(local)
    from iceicle_b200.partition import StripPlan, StripResidual
    from iceicle_b200.workloads import ns_mms_config, ns_mms_strip_config
    if ws > 1:
        # weak scaling over element-row strips: rank r owns rows
        # [128 r, 128 (r + 1)) of the 128 x 128 ws mesh plus one ghost row per
        # neighbour; a step is the halo exchange (NCCL send/recv of one row of
        # coefficients per neighbour) and the residual of the rank's sub-mesh
        plan = StripPlan(NX, NY * ws, ws, rank, 2)
        wl = ns_mms_strip_config(plan, p=3, geo_order=2, device=local)
        step_fn = StripResidual(wl.ctx, plan)
        o0, o1 = plan.owned_dofs(wl.ctx.layout.block_size)
    else:
        plan = None
        wl = ns_mms_config(nx=NX, ny=NY, p=3, geo_order=2, device=local)
        step_fn = wl.ctx.form_residual
        o0, o1 = 0, wl.ctx.layout.n_dof
    N = o1 - o0  # owned DOFs of this rank
    dev = torch.device("cuda", local)
    u = torch.from_numpy(wl.u0).to(dev)
    res = torch.empty_like(u)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    # launch shapes of the face and volume kernels for this (p, neq), chosen
    # once before any timing (every shape computes identical values)
    import iceicle_b200 as ib
    tune = None
    if a.tile:
        wl.ctx.tile = {k: int(v) for k, v in (kv.split("=") for kv in a.tile.split(","))}
    elif not a.no_tune:
        tune = wl.ctx.autotune(u, ib.TUNE_RESIDUAL)
    for _ in range(max(a.warmup, 3)):
        step_fn(u, res, stream)
    torch.cuda.synchronize(dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    sampler = ClockSampler(local)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for k in range(a.steps):
        flush.zero_()
        starts[k].record(stream)
        step_fn(u, res, stream)
        ends[k].record(stream)
    torch.cuda.synchronize(dev)
    if ws > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    # per-kernel split (events around each kernel on the same stream)
    t_face, t_vol = [], []
    for _ in range(max(3, min(a.steps, 10))):
        flush.zero_()
        f, v = wl.ctx.form_residual_timed(u, res, stream)
        t_face.append(f)
        t_vol.append(v)
    # end to end through the public API with host buffers: one state per step,
    # copied in from pinned host memory and its residual copied back
    # (icx_form_residuals_host overlaps the copies of consecutive steps); the
    # same measured one step at a time, each step's copies and kernels in turn
    # (with strips: each step copies the rank's owned rows in, exchanges the
    # halo and copies the owned residual back, one step at a time)
    if plan is None:
        h_u = torch.from_numpy(np.tile(wl.u0, (a.steps, 1))).pin_memory()
        h_r = torch.empty((a.steps, N), dtype=torch.float64).pin_memory()
        for _ in range(max(a.warmup, 3) // 3):  # warm-up over the same host buffers (first touches from the GPU)
            wl.ctx.form_residuals_host(h_u, h_r)
        torch.cuda.synchronize(dev)
        ms_e2e = wl.ctx.form_residuals_host(h_u, h_r)
        h_u1, h_r1 = h_u[0], h_r[0]
    else:
        h_u1 = torch.from_numpy(wl.u0[o0:o1].copy()).pin_memory()
        h_r1 = torch.empty(N, dtype=torch.float64).pin_memory()
    e2e_s = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    e2e_e = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    for k in range(-1, a.steps):  # one untimed step first
        flush.zero_()
        if k >= 0:
            e2e_s[k].record(stream)
        u[o0:o1].copy_(h_u1, non_blocking=True)
        step_fn(u, res, stream)
        h_r1.copy_(res[o0:o1], non_blocking=True)
        if k >= 0:
            e2e_e[k].record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e_seq = sum(s.elapsed_time(e) for s, e in zip(e2e_s, e2e_e))
    if plan is not None:
        ms_e2e = ms_e2e_seq
    if ws > 1:
        t = torch.tensor([ms, ms_e2e, ms_e2e_seq], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_e2e_seq = t.tolist()
    if rank == 0:
        value = ws * N * a.steps / (ms * 1e-3)
        e2e = ws * N * a.steps / (ms_e2e * 1e-3)
        e2e_seq = ws * N * a.steps / (ms_e2e_seq * 1e-3)
        work = residual_work(wl)
        tv = float(np.median(t_vol)) * 1e-3
        tf = float(np.median(t_face)) * 1e-3
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        hbm = peaks.get("hbm_gbs", 6650.0)
        dom = "vol" if tv >= tf else "face"
        shape = wl.ctx.tile  # 0: the compiled default (face bound 5; volume 256 threads, bound 4)
        shape = {"face_minb": shape["face_minb"] or 5, "vol_threads": shape["vol_threads"] or 256,
                 "vol_minb": shape["vol_minb"] or 4}
        td = tv if dom == "vol" else tf
        bytes_d, flops_d = work[dom]
        achieved = bytes_d / td / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded manufactured solution)",
            "config": WORKLOAD,
            "parallelism": (f"element-row strips x{ws}: 128 x 128 owned per GPU of a 128 x {NY * ws} mesh, "
                            "one halo row per neighbour (NCCL send/recv)") if ws > 1 else "single GPU",
            "e2e": {"value": e2e, "unit": "DOF/s", "h2d_bytes_per_step": 8 * N, "d2h_bytes_per_step": 8 * N,
                    "api": ("icx_form_residuals_host (copies of consecutive steps overlapped)" if ws == 1 else
                            "owned rows in, halo exchange, icx_form_residual, owned residual out; one step at a time"),
                    "one_step_at_a_time": e2e_seq},
            "gpu_launches": 2 * a.steps,
            "roofline": {"bound": "hbm",
                         "kernel": (f"vol_lift_kernel<NS,p3,g2> ({shape['vol_threads']} threads, "
                                    f"{shape['vol_minb']} CTAs/SM bound)") if dom == "vol" else
                                   f"face_flux_kernel<NS,p3,g2,IP> ({shape['face_minb']} CTAs/SM bound)",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                         else "fallback 6650 GB/s",
                         "traffic": NCU_DRAM_BYTES[dom], "algorithmic_bytes": bytes_d,
                         "kernel_ms": {"face_flux": tf * 1e3, "vol_lift": tv * 1e3},
                         "fp64": {"flops_per_launch": flops_d, "achieved_tflops": flops_d / td / 1e12,
                                  "nominal_peak_tflops": 37.0},
                         "other_kernel": {"name": "face_flux" if dom == "vol" else "vol_lift",
                                          "algorithmic_bytes": work["face" if dom == "vol" else "vol"][0],
                                          "achieved_gbs": work["face" if dom == "vol" else "vol"][0] /
                                          (tf if dom == "vol" else tv) / 1e9}},
            "clocks": clocks,
            "autotune": {"fixed": {k: wl.ctx.tile[k] for k in ("face_minb", "vol_threads", "vol_minb")}}
            if tune is None else {
                "chosen": {k: tune["chosen"][k] for k in ("face_minb", "vol_threads", "vol_minb")},
                "residual_ms_default": tune["residual_ms_default"], "residual_ms_tuned": tune["residual_ms_tuned"],
                "shapes_timed": tune["n_timed"], "rejected": tune["n_rejected"]},
        }
        if not a.no_cpu_baseline and ws == 1:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            import oracle_bindings as ob
            if ob.ref_available():
                n, t, _ = _ref_worker((3, 0))
                line["cpu_baseline"] = {"value": n / t, "unit": "DOF/s", "cores": 1, "kind": "reference",
                                        "sample": "3 full 128x128 p3 residuals, 1 thread (reference is serial)"}
            else:
                line["cpu_baseline"] = None
        wall = {}

        def section(name, fn):
            t0 = time.time()
            line[name] = fn()
            wall[name] = round(time.time() - t0, 1)
        if ws == 1:
            section("residual_roe", lambda: roe_residual_bench(torch, dev, flush, tune is not None))
            section("jacobian", lambda: jacobian_bench(torch, dev, wl, hbm, not a.no_cpu_baseline))
        if not a.no_newton and ws == 1:
            section("newton", lambda: newton_bench(torch, dev, not a.no_tune))
            if not a.no_lm:
                section("mdg_ice", lambda: lm_bench(torch, dev))
        if a.batched and ws == 1:
            section("batched", lambda: batched_bench(torch, dev, a.batched, a.batched_sample, a.batched_fp32q))
        if not a.no_learned and ws == 1:
            section("learned_pc", lambda: learned_bench(torch, dev, not a.no_tune, a.learned_seeds))
        line["section_wall_s"] = wall
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()


def gemm_mode(spec):
    """tcgen05 BF16 GEMM alone: 20 launches after 3 untimed, CUDA events,
    2 M N K flops per launch against the measured dense BF16 peak"""
    import torch
    import iceicle_b200 as ib
    M, N, K = (int(v) for v in spec.split(","))
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C32 = torch.empty(M, N, device="cuda", dtype=torch.float32)
    for _ in range(3):
        ib.gemm_bf16_nt(A, B, out32=C32)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(20):
        ib.gemm_bf16_nt(A, B, out32=C32)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 20
    ref = (A.float() @ B.float().T)
    err = float((C32 - ref).abs().max() / ref.abs().max())
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("bf16_tflops", 1590.0)
    tf = 2.0 * M * N * K / (ms * 1e-3) / 1e12
    print(json.dumps({"mode": "gemm_bf16_nt", "M": M, "N": N, "K": K, "ms": ms, "tflops": tf, "peak_tflops": peak,
                      "frac": tf / peak, "max_rel_err_vs_fp32_of_bf16_inputs": err}))


def jacobian_mode(n):
    """the FD Jacobian alone on the n x n p = 3 Navier-Stokes workload: FP64
    and FP32 flux quadrature, mean of 5 launches after 2 untimed (CUDA events)"""
    import torch
    from iceicle_b200.workloads import ns_mms_config
    wl = ns_mms_config(nx=n, ny=n, p=3, geo_order=2)
    L = wl.ctx.layout
    bs = L.block_size
    u = torch.from_numpy(wl.u0).cuda()
    res = torch.empty_like(u)
    out = {"mode": "jacobian_fd", "mesh": f"{n}x{n}", "p": 3, "n_dof": L.n_dof}
    for name, dt, fn in (("fp64", torch.float64, wl.ctx.form_jacobian_fd),
                         ("fp32_quadrature", torch.float32, wl.ctx.form_jacobian_fd_f32)):
        vals = torch.empty(L.nnz_blocks * bs * bs, dtype=dt, device="cuda")
        for _ in range(2):
            fn(u, res, vals)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(5):
            fn(u, res, vals)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 5
        written = vals.numel() * vals.element_size()
        out[name] = {"ms_with_residual": ms, "bsr_bytes": written, "gbs_written": written / (ms * 1e-3) / 1e9}
        del vals
    print(json.dumps(out))


def solve_mode(tile, precision, matrix_free=0):
    """one Newton solve (|r| <= 1e-10, GMRES(30)) of the first evaluation
    instance of the 256 x 256 p = 2 Navier-Stokes problem, launch shapes
    autotuned at the initial state for the chosen tiling; CUDA events around
    the solve"""
    import torch
    import iceicle_b200 as ib
    from iceicle_b200 import learned_pc as lp
    dev = torch.device("cuda", 0)
    seed, re = lp.instances(*lp.EVAL_INSTANCES)[0]
    wl = lp.make_instance(seed, re, 256, dev.index)
    u0 = torch.from_numpy(wl.u0).to(dev)
    wl.ctx.ilu_tile = tile
    wl.ctx.autotune(u0, ib.TUNE_RESIDUAL | ib.TUNE_ILU | ib.TUNE_ILU_FP32)
    opt = ib.default_newton_options()
    opt.precision, opt.ilu_tile, opt.gmres_max_it, opt.matrix_free = precision, tile, 20000, matrix_free
    opt.gmres_cgs_refine = 0  # PETSc's default GMRES orthogonalisation
    u = u0.clone()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    rep = wl.ctx.newton_solve(u, opt)
    e1.record()
    torch.cuda.synchronize(dev)
    s = e0.elapsed_time(e1) * 1e-3
    its = rep.linear_iterations_total
    print(json.dumps({"solve": "ns_256x256_p2", "seed": seed, "re": re, "ilu_tile": tile, "precision": precision,
                      "matrix_free": matrix_free,
                      "converged": bool(rep.converged), "s": s, "newton_its": rep.iterations, "gmres_its": its,
                      "ms_per_gmres_it": 1e3 * s / max(its, 1), "tile_choice": wl.ctx.tile}))


def main():
    a = parse()
    if a.solve >= 0:
        solve_mode(a.solve, a.solve_precision, int(a.solve_matrix_free))
        return
    if a.gemm:
        gemm_mode(a.gemm)
        return
    if a.jacobian:
        jacobian_mode(a.jacobian)
        return
    if a.spmv:
        spmv_bench(a.spmv)
    elif a.ilu:
        ilu_bench(a.ilu)
    elif a.factor:
        factor_bench()
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
