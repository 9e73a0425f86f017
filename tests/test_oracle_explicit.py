"""Explicit time stepping on the oracle, pinned to the reference's own
ExplicitEuler / RK3TVD / RK3SSP (explicit_euler.hpp, tvd_rk3.hpp,
ssp_rk3.hpp) and calculate_mass_matrix (finite_element.hpp:587-610) compiled
in the reference build. CPU only."""
import numpy as np
import pytest

import oracle_bindings as ob
from specs import BURGERS, NS, Spec

pytestmark = pytest.mark.skipif(not ob.ref_available(), reason="reference build oracle/_ref not present")

MASS_CASES = [dict(nx=3, ny=2, g=1, p=1, perturb=0.0), dict(nx=3, ny=3, g=2, p=2), dict(nx=2, ny=2, g=2, p=4)]


@pytest.mark.parametrize("kw", MASS_CASES, ids=[str(c) for c in MASS_CASES])
def test_mass_matrices_match_reference(kw):
    spec = Spec(**kw)
    c = spec.coords()
    pb = spec.oracle_problem()
    Mo = ob.mass_matrices(ob.oracle(), pb, c)
    Mr = ob.mass_matrices(ob.ref(), pb, c)
    assert np.abs(Mo - Mr).max() <= 1e-14 * np.abs(Mr).max()


# (scheme, dt_kind, dt, cfl, term_kind, ntime, tfinal)
RUNS = [
    (0, 0, 2e-3, 0.0, 0, 3, 0.0),
    (1, 0, 2e-3, 0.0, 0, 3, 0.0),
    (2, 0, 2e-3, 0.0, 0, 3, 0.0),
    (0, 1, 0.0, 0.3, 0, 4, 0.0),
    (1, 1, 0.0, 0.3, 1, 0, 0.01),
    (2, 1, 0.0, 0.5, 1, 0, 0.01),
]


@pytest.mark.parametrize("run", RUNS, ids=[str(r) for r in RUNS])
def test_explicit_burgers_matches_reference(run):
    spec = Spec(pde=BURGERS, nx=3, ny=3, g=2, p=2, mu=0.01, a=(0.3, -0.2), b=(1.0, 0.5))
    c = spec.coords()
    pb = spec.oracle_problem()
    u0 = spec.state(np.random.default_rng(3))
    scheme, dk, dt, cfl, tk, nt, tf = run
    uo, so, to = ob.explicit_solve(ob.oracle(), pb, c, u0, scheme, dk, dt, cfl, tk, nt, tf)
    ur, sr, tr = ob.explicit_solve(ob.ref(), pb, c, u0, scheme, dk, dt, cfl, tk, nt, tf)
    assert so == sr and abs(to - tr) <= 1e-14 * max(tr, 1.0)
    assert np.abs(uo - ur).max() <= 1e-12 * np.abs(ur).max()
    assert np.abs(uo - u0).max() > 0.0


def test_explicit_ns_tvd_matches_reference():
    spec = Spec(pde=NS, nx=2, ny=2, g=2, p=2, ip=True, source=True, perturb=0.05)
    c = spec.coords()
    pb = spec.oracle_problem()
    u0 = spec.state(np.random.default_rng(4))
    uo, _, _ = ob.explicit_solve(ob.oracle(), pb, c, u0, 1, 0, 1e-4, 0.0, 0, 2, 0.0)
    ur, _, _ = ob.explicit_solve(ob.ref(), pb, c, u0, 1, 0, 1e-4, 0.0, 0, 2, 0.0)
    assert np.abs(uo - ur).max() <= 1e-12 * np.abs(ur).max()


def test_ssp_rk3_stages_use_the_step_start_state():
    """the reference's SSP-RK3 evaluates every stage residual at the state the
    step starts from, so one step equals the Euler step dt * (1/6 + 1/6 + 2/3)
    M^-1 R(u) (up to rounding of the three updates)"""
    spec = Spec(pde=BURGERS, nx=3, ny=2, g=1, p=1, perturb=0.0)
    c = spec.coords()
    pb = spec.oracle_problem()
    u0 = spec.state(np.random.default_rng(5))
    us, _, _ = ob.explicit_solve(ob.ref(), pb, c, u0, 2, 0, 1e-3, 0.0, 0, 1, 0.0)
    ue, _, _ = ob.explicit_solve(ob.ref(), pb, c, u0, 0, 0, 1e-3, 0.0, 0, 1, 0.0)
    assert np.abs(us - ue).max() <= 1e-14 * np.abs(ue).max()
