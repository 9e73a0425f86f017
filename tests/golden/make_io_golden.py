"""Writes the restart and VTU golden files under tests/golden/io/ with the
reference's own writers (write_restart, PVDWriter::write_vtu and the MDG
residual writer of its implicit driver), compiled into
oracle/_ref/libiceicle_ref.so. Run from the repository root:

    python tests/golden/make_io_golden.py

The cases are seeded and small; IO_CASES is shared with the tests that read
the files."""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle_bindings as ob  # noqa: E402
from specs import BURGERS, NS, Spec  # noqa: E402

GOLDEN_IO = os.path.join(HERE, "io")

# name -> (Spec keywords, state seed, restart index k, VTU itime, MDG traces)
IO_CASES = {
    "burgers_3x2_p2_g2": (dict(pde=BURGERS, nx=3, ny=2, g=2, p=2, mu=1e-2, a=(0.3, -0.2), b=(1.0, 0.5)),
                          11, 3, 5, None),
    "burgers_3x3_p1_g1": (dict(pde=BURGERS, nx=3, ny=3, g=1, p=1, mu=0.02), 12, 0, 2, None),
    "ns_2x2_p3_g2": (dict(pde=NS, nx=2, ny=2, g=2, p=3, ip=True, perturb=0.05), 13, 7, 1, None),
    "mdg_4x4_p2_g1": (dict(pde=BURGERS, nx=4, ny=4, g=1, p=2, mu=0.0, a=(0.0, 1.0), b=(1.0, 0.0),
                           bct=(3, 3, 3, 4), dirichlet=[("oblique_step", [0.4, 0.2, 1.0, -0.5])]),
                      14, 1, 4, "interior"),
}


def case_inputs(name):
    """(spec, coords, state, k, itime, traces, ic) of a case; ic is the seeded
    interface residual of the selected nodes (MDG cases) or None"""
    kw, seed, k, itime, traces = IO_CASES[name]
    spec = Spec(**kw)
    c = spec.coords()
    u = spec.state(np.random.default_rng(seed))
    tr, ic = None, None
    if traces == "interior":
        pb = spec.oracle_problem()
        _, _, nint = ob.topology(ob.oracle(), pb)
        tr = np.arange(nint)
        sel, _ = ob.mdg_select(ob.oracle(), pb, c, tr)
        ic = np.random.default_rng(seed + 100).standard_normal(len(sel) * spec.neq)
    return spec, c, u, k, itime, tr, ic


def main():
    if os.path.isdir(GOLDEN_IO):
        shutil.rmtree(GOLDEN_IO)
    for name in IO_CASES:
        spec, c, u, k, itime, tr, ic = case_inputs(name)
        pb = spec.oracle_problem()
        d = os.path.join(GOLDEN_IO, name)
        os.makedirs(d)
        ob.ref_write_restart(pb, c, u, k, d)
        ob.ref_write_vtu(pb, c, u, 0, itime, d, "data")
        ob.ref_write_vtu(pb, c, u, 1, itime, d, "residuals")
        if ic is not None:
            ob.ref_write_vtu_mdg(pb, c, tr, True, ic, itime, d, "mdg_residuals")
    print("wrote", GOLDEN_IO)


if __name__ == "__main__":
    main()
