"""The C++23 facade (include/iceicle_b200.hpp) run on the GPU: the program
tests/cpp/facade_check.cpp, compiled here with g++ and linked against the
product library, uses ConservationLawDDG with the reference's flux objects,
form_residual, form_jacobian_fd and NewtonSolver. Its printed results are
compared with the oracle on the same meshes and states: residuals at 1e-12 of
the largest entry, the Newton state with the oracle Newton's at 1e-10."""
import os
import subprocess

import numpy as np
import pytest

import oracle_bindings as ob
import oracle_newton as on
from specs import BURGERS, NS, Spec
from test_cpp_facade import build_facade_check

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def facade_run(tmp_path_factory):
    d = tmp_path_factory.mktemp("facade")
    exe = str(d / "facade_check")
    r = build_facade_check(exe)
    assert r.returncode == 0, r.stderr[-4000:]
    b_spec = Spec(pde=BURGERS, nx=4, ny=3, p=2, g=2, perturb=0.0, mu=0.01, a=(0.3, -0.2), b=(1.0, 0.5),
                  dirichlet=[("constant", [1, 0.25])])
    u_b = b_spec.state(np.random.default_rng(31))
    n_spec = Spec(pde=NS, nx=3, ny=3, p=2, g=2, perturb=0.0, ip=True, ns_flux=2, bct=(5, 7, 5, 6), bcf=(0, 0, 0, 1),
                  walls=(0.004, 0.005), free_stream=(1.0, 0.5, (1.0, 0.0), 0.004), sutherland=(0.02, 0.004, 0.0015))
    u_n = n_spec.state(np.random.default_rng(32))
    np.savetxt(d / "ub.txt", u_b)
    np.savetxt(d / "un.txt", u_n)
    out = subprocess.run([exe, str(d / "ub.txt"), str(d / "un.txt")], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-4000:]
    lines = {ln.split()[0]: ln.split()[1:] for ln in out.stdout.splitlines() if ln.strip()}
    return lines, (b_spec, u_b), (n_spec, u_n)


def _vec(fields):
    n = int(fields[0])
    v = np.array([float(x) for x in fields[1:]])
    assert v.size == n
    return v


def test_facade_burgers_residual(facade_run):
    lines, (spec, u), _ = facade_run
    r = _vec(lines["residual"])
    ref = ob.residual(ob.oracle(), spec.oracle_problem(), spec.coords(), u)
    assert np.abs(r - ref).max() <= 1e-12 * np.abs(ref).max()
    nnzb, bs = (int(x) for x in lines["jacobian_blocks"])
    assert bs == 9 and nnzb == 4 * 3 + 2 * ((4 - 1) * 3 + 4 * (3 - 1))
    assert float(lines["jacobian_f32_rel"][0]) <= 2e-3  # FP32 flux quadrature against the FP64 blocks


def test_facade_ns_roe_wall_residual(facade_run):
    lines, _, (spec, u) = facade_run
    r = _vec(lines["ns_residual"])
    ref = ob.residual(ob.oracle(), spec.oracle_problem(), spec.coords(), u)
    assert np.abs(r - ref).max() <= 1e-12 * np.abs(ref).max()


def test_facade_newton_matches_oracle_newton(facade_run):
    lines, _, _ = facade_run
    its, rfin = int(lines["newton"][0]), float(lines["newton"][1])
    assert rfin <= 1e-10 and its >= 2
    u = _vec(lines["newton_state"])
    spec = Spec(pde=BURGERS, nx=8, ny=8, p=2, g=2, perturb=0.0, mu=0.01, a=(0.0, 0.0), b=(1.0, 0.5),
                dirichlet=[("constant", [1, 0.0])])
    c = spec.coords()
    pb = spec.oracle_problem()
    xy = ob.basis_node_coords(pb, c)
    u0 = (np.sin(2 * np.pi * xy[..., 0]) * np.sin(2 * np.pi * xy[..., 1])).reshape(-1)
    u_or, hist = on.newton(pb, c, u0, tau_abs=1e-10, kmax=20, linesearch="wolfe")
    assert hist[-1] <= 1e-10
    # the steady state is u = 0: the state difference is measured against the initial state's norm
    assert np.linalg.norm(u - u_or) <= 1e-10 * max(np.linalg.norm(u_or), np.linalg.norm(u0))
