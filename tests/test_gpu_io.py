"""Restart files and VTU output written from the GPU state (C ABI) against the
reference's own writers: the golden files under tests/golden/io, made by the
reference build (tests/golden/make_io_golden.py)."""
import os
import sys

import numpy as np
import pytest
import torch

import iceicle_b200 as ib
from io_files import vtu_diff

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_io_golden import GOLDEN_IO, IO_CASES, case_inputs  # noqa: E402

pytestmark = pytest.mark.gpu


def _read(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("name", list(IO_CASES))
def test_restart_file_matches_the_reference_byte_for_byte(name, tmp_path):
    spec, c, u, k, itime, tr, ic = case_inputs(name)
    ctx = spec.context(c)
    ctx.write_restart(torch.from_numpy(u).cuda(), k, 0, tmp_path / "RESTART")
    assert _read(tmp_path / "RESTART" / f"restart{k}_0") == _read(
        os.path.join(GOLDEN_IO, name, "RESTART", f"restart{k}_0"))


@pytest.mark.parametrize("name", list(IO_CASES))
def test_read_restart_moves_the_mesh_and_restores_the_state(name):
    """a context built on the unperturbed lattice reads the reference's file:
    its nodes and state become the file's (16 significant digits, 1e-15
    relative), and its residual is then bit-identical to that of a context
    built on the same coordinates (the geometry is recomputed)"""
    spec, c, u, k, itime, tr, ic = case_inputs(name)
    from iceicle_b200.workloads import lattice_coords
    ctx = spec.context(lattice_coords((spec.nx, spec.ny), spec.g))
    du = torch.zeros(spec.N, dtype=torch.float64, device="cuda")
    ctx.read_restart(du, f"restart{k}", 0, os.path.join(GOLDEN_IO, name, "RESTART"))
    xy = ctx.get_coords().reshape(-1)
    assert np.allclose(xy, c.reshape(-1), rtol=1e-15, atol=1e-16)
    assert np.allclose(du.cpu().numpy(), u, rtol=1e-15, atol=1e-16)
    ctx2 = spec.context(xy.reshape(-1, 2).copy())
    r1, r2 = torch.empty_like(du), torch.empty_like(du)
    ctx.form_residual(du, r1)
    ctx2.form_residual(du, r2)
    torch.cuda.synchronize()
    assert torch.equal(r1, r2)


@pytest.mark.parametrize("name", list(IO_CASES))
@pytest.mark.parametrize("kind,coll", [(ib.VTU_SOLUTION, "data"), (ib.VTU_RESIDUAL, "residuals")])
def test_vtu_matches_the_reference(name, kind, coll, tmp_path):
    """tags, names, connectivity, offsets and cell types identical; point
    coordinates, fields and residuals (full, domain_, trace_) to 1e-6 of each
    array's largest value, 8 significant digits being printed"""
    spec, c, u, k, itime, tr, ic = case_inputs(name)
    ctx = spec.context(c)
    ctx.write_vtu(torch.from_numpy(u).cuda(), itime, kind, tmp_path)
    f = f"{coll}{itime}.vtu"
    d = vtu_diff(_read(tmp_path / f).decode(), _read(os.path.join(GOLDEN_IO, name, f)).decode())
    assert d is None, d


def test_mdg_residual_vtu_matches_the_reference(tmp_path):
    name = "mdg_4x4_p2_g1"
    spec, c, u, k, itime, tr, ic = case_inputs(name)
    ctx = spec.context(c)
    ctx.mdg_select(tr, True)
    ctx.write_vtu_mdg(torch.from_numpy(ic).cuda(), itime, tmp_path)
    f = f"mdg_residuals{itime}.vtu"
    d = vtu_diff(_read(tmp_path / f).decode(), _read(os.path.join(GOLDEN_IO, name, f)).decode())
    assert d is None, d


def test_restart_round_trip_through_the_library(tmp_path):
    spec, c, u, k, itime, tr, ic = case_inputs("ns_2x2_p3_g2")
    ctx = spec.context(c)
    du = torch.from_numpy(u).cuda()
    ctx.write_restart(du, 9, 2, tmp_path)
    back = torch.zeros_like(du)
    ctx.read_restart(back, "restart9", 2, tmp_path)
    assert np.allclose(back.cpu().numpy(), u, rtol=1e-15, atol=1e-16)


def test_io_errors_are_reported(tmp_path):
    spec, c, u, k, itime, tr, ic = case_inputs("burgers_3x3_p1_g1")
    ctx = spec.context(c)
    du = torch.from_numpy(u).cuda()
    with pytest.raises(ib.IcxError) as e:
        ctx.read_restart(du, "missing", 0, tmp_path)
    assert e.value.status == 1
    (tmp_path / "short_0").write_text("0 0 1 0 \n1 2 3")
    with pytest.raises(ib.IcxError) as e:
        ctx.read_restart(du, "short", 0, tmp_path)
    assert e.value.status == 1
    with pytest.raises(ib.IcxError) as e:
        ctx.write_vtu_mdg(du, 0, tmp_path)  # no node selection
    assert e.value.status == 1
    b = ib.batch([ctx, spec.context(c)])
    with pytest.raises(ib.IcxError) as e:
        b.write_restart(torch.cat([du, du]), 0, 0, tmp_path)
    assert e.value.status == 3
