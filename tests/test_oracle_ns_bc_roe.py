"""Navier-Stokes PDE-level boundaries and the Roe flux on the oracle side (CPU).

* The wall and characteristic boundaries (apply_bc, navier_stokes.hpp:976-1189:
  slip wall, no-slip isothermal wall, WALL_GENERAL, Riemann) are pinned to the
  reference's own code compiled here: residuals to 1e-12 of the largest entry.
* The Roe flux has no reference counterpart (parity unpinned): it is checked
  for consistency as the reference checks its Van Leer flux
  (test/test_ns.cpp:67-107: F(u, u, n) = F(u) . n to 1e-10 for the states
  rho = 1, v = (s, s), rho E = 1.4 with s in {-1, -0.001, 0, 0.001, 1}), for
  conservation (F(uL, uR, n) = -F(uR, uL, -n)) and for upwinding (a
  supersonic state crossing a face is carried by its upwind side)."""
import ctypes as C

import numpy as np
import pytest

import oracle_bindings as ob
from specs import NS, Spec

needs_ref = pytest.mark.skipif(not ob.ref_available(), reason="reference CPU build absent")

WALL_T = (0.004, 0.005)
FREE = (1.0, 0.5, (1.0, 0.0), 0.004)

BC_CASES = [
    dict(pde=NS, p=2, ip=True, bct=(5, 7, 5, 6), bcf=(0, 0, 0, 1), walls=WALL_T, free_stream=FREE),
    dict(pde=NS, p=1, g=1, bct=(8, 8, 8, 8), walls=WALL_T[:1]),
    dict(pde=NS, p=3, bct=(6, 5, 7, 3), bcf=(1, 0, 0, 0), walls=WALL_T, free_stream=(1.2, 0.3, (0.6, 0.8), 0.0035)),
    dict(pde=NS, p=2, ns_mu=0.0, bct=(8, 5, 8, 5), free_stream=FREE),  # inviscid: WALL_GENERAL is the slip wall
    dict(pde=NS, p=2, bct=(5, 5, 5, 5), free_stream=(1.0, 2.5, (0.0, 1.0), 0.004)),  # supersonic free stream
]


@needs_ref
@pytest.mark.parametrize("kw", BC_CASES, ids=[str(i) for i in range(len(BC_CASES))])
def test_ns_pde_boundaries_match_reference(kw):
    spec = Spec(**kw)
    pb = spec.oracle_problem()
    c = spec.coords()
    u = spec.state(np.random.default_rng(4))
    r_or = ob.residual(ob.oracle(), pb, c, u)
    r_ref = ob.residual(ob.ref(), pb, c, u)
    assert np.abs(r_or - r_ref).max() <= 1e-12 * np.abs(r_ref).max()


def _flux_fns():
    lib = ob.oracle().lib
    f = lib.orc_numerical_flux
    f.argtypes = [C.c_void_p] * 5
    g = lib.orc_physical_flux
    g.argtypes = [C.c_void_p] * 4
    return f, g


def _num(pb, uL, uR, n):
    f, _ = _flux_fns()
    out = np.zeros(4)
    f(C.addressof(pb), ob._ptr(np.ascontiguousarray(uL, float)), ob._ptr(np.ascontiguousarray(uR, float)),
      ob._ptr(np.ascontiguousarray(n, float)), ob._ptr(out))
    return out


def _phys(pb, u):
    _, g = _flux_fns()
    F = np.zeros((4, 2))
    g(C.addressof(pb), ob._ptr(np.ascontiguousarray(u, float)), ob._ptr(np.zeros(8)), ob._ptr(F))
    return F


@pytest.mark.parametrize("flux", [1, 2], ids=["van_leer", "roe"])
def test_numerical_flux_consistency(flux):
    pb = Spec(pde=NS, ns_flux=flux).oracle_problem()
    for s in (-1.0, -0.001, 0.0, 0.001, 1.0):
        u = np.array([1.0, s, s, 1.4])
        F = _phys(pb, u)
        for n in ((1.0, 0.0), (0.0, 1.0), (0.6, -0.8)):
            fn = _num(pb, u, u, n)
            np.testing.assert_allclose(fn, F @ np.array(n), rtol=0, atol=1e-10)


def test_roe_flux_conservation_and_upwinding():
    pb = Spec(pde=NS, ns_flux=2).oracle_problem()
    rng = np.random.default_rng(3)
    for _ in range(20):
        uL = np.array([1.0, 0.3, -0.2, 2.5]) * (1 + 0.2 * rng.standard_normal(4))
        uR = np.array([0.8, -0.1, 0.4, 2.0]) * (1 + 0.2 * rng.standard_normal(4))
        th = rng.uniform(0, 2 * np.pi)
        n = np.array([np.cos(th), np.sin(th)])
        np.testing.assert_allclose(_num(pb, uL, uR, n), -_num(pb, uR, uL, -n), rtol=1e-12, atol=1e-13)
    # supersonic flow along +x (Mach ~ 2.6): the flux is the left state's physical flux
    uL = np.array([1.0, 3.0, 0.0, 1.0 / 0.4 + 4.5])
    uR = np.array([0.7, 2.0, 0.1, 1.5 / 0.4 + 0.5 * (4 + 0.01) / 0.7])
    n = np.array([1.0, 0.0])
    np.testing.assert_allclose(_num(pb, uL, uR, n), _phys(pb, uL) @ n, rtol=1e-12, atol=1e-12)
