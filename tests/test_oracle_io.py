"""The restart and VTU golden files against the reference's own writers
(compiled into oracle/_ref), and the reference's restart reader on them."""
import os
import sys

import numpy as np
import pytest

import oracle_bindings as ob

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_io_golden import GOLDEN_IO, IO_CASES, case_inputs  # noqa: E402

needs_ref = pytest.mark.skipif(not ob.ref_available(), reason="reference CPU build absent")


def _read(path):
    with open(path, "rb") as f:
        return f.read()


@needs_ref
@pytest.mark.parametrize("name", list(IO_CASES))
def test_golden_files_are_what_the_reference_writes(name, tmp_path):
    """regenerating a case with the reference's writers reproduces the
    committed files byte for byte"""
    spec, c, u, k, itime, tr, ic = case_inputs(name)
    pb = spec.oracle_problem()
    ob.ref_write_restart(pb, c, u, k, tmp_path)
    ob.ref_write_vtu(pb, c, u, 0, itime, tmp_path, "data")
    ob.ref_write_vtu(pb, c, u, 1, itime, tmp_path, "residuals")
    files = [f"RESTART/restart{k}_0", f"data{itime}.vtu", f"residuals{itime}.vtu"]
    if ic is not None:
        ob.ref_write_vtu_mdg(pb, c, tr, True, ic, itime, tmp_path, "mdg_residuals")
        files.append(f"mdg_residuals{itime}.vtu")
    for f in files:
        assert _read(tmp_path / f) == _read(os.path.join(GOLDEN_IO, name, f)), f


@needs_ref
@pytest.mark.parametrize("name", list(IO_CASES))
def test_reference_reads_back_the_golden_restart(name):
    """read_restart on the golden file returns the coordinates and state that
    were written (16 significant digits: 1e-15 relative)"""
    spec, c, u, k, itime, tr, ic = case_inputs(name)
    pb = spec.oracle_problem()
    c2, u2 = ob.ref_read_restart(pb, f"restart{k}", os.path.join(GOLDEN_IO, name))
    assert np.allclose(c2, c.reshape(-1), rtol=1e-15, atol=1e-16)
    assert np.allclose(u2, u, rtol=1e-15, atol=1e-16)


def test_golden_restart_layout():
    """node coordinates on the first line, then nb*neq values per element"""
    for name in IO_CASES:
        spec, c, u, k, itime, tr, ic = case_inputs(name)
        with open(os.path.join(GOLDEN_IO, name, "RESTART", f"restart{k}_0")) as f:
            first, rest = f.read().split("\n", 1)
        assert len(first.split()) == c.size
        assert len(rest.split()) == spec.N
