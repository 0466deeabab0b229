"""The output path of runTimeLoop on the CPU: the VTK writer of the CUDA
library (sifv_vtk_*, host only) against the reference's own runTimeLoop +
VTKSession byte for byte, with the oracle stepping the same problem, and the
oracle's NaN check against the rule it restates."""
import filecmp
import os

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi


def _tree(root):
    out = {}
    for d, _, files in os.walk(root):
        for f in files:
            p = os.path.join(d, f)
            out[os.path.relpath(p, root)] = p
    return out


def assert_same_tree(a, b):
    ta, tb = _tree(a), _tree(b)
    assert sorted(ta) == sorted(tb)
    for rel in ta:
        assert filecmp.cmp(ta[rel], tb[rel], shallow=False), rel


def loop_case(name):
    """(case, end_time, output_interval) with a handful of steps and an
    interval that does not divide the end time."""
    if name == "sod":
        case = cases.sod(64)
    elif name == "riemann2d":
        case = cases.riemann2d(20, bc=abi.BC_SLIPWALL)
    elif name == "water_air":
        case = cases.water_air(48)
    elif name == "acoustic3d_igr":
        case = cases.acoustic3d(6)
    elif name == "droplet2d":
        case = cases.droplet(16)
    else:
        raise KeyError(name)
    probe = backends.make(backends.oracle(), case)
    dt0 = probe.step(0, 0.0, -1.0)
    return case, 5.5 * dt0, 2.2 * dt0


LOOP_CASES = ["sod", "riemann2d", "water_air", "acoustic3d_igr", "droplet2d"]


@pytest.mark.parametrize("name", LOOP_CASES)
def test_vtk_files_match_reference_time_loop(name, tmp_path):
    ref = backends.reference()
    if ref is None:
        pytest.skip("reference not built")
    case, t_end, every = loop_case(name)
    cr = backends.make(ref, case)
    steps_ref = cr.reference_time_loop(str(tmp_path / "ref"), name, t_end, every)

    co = backends.make(backends.oracle(), case)
    vtk = abi.VtkSession(backends.cuda(), str(tmp_path / "ours"), name, case[0], case[1], threads=3)
    _, steps = cases.run_time_loop(co, t_end, every,
                                   on_output=lambda t, s: vtk.write_host(t, cases.output_fields(co, case[0])))
    vtk.close()
    assert steps == steps_ref
    assert_same_tree(str(tmp_path / "ref"), str(tmp_path / "ours"))


def test_vtk_number_format_is_printf_g15(tmp_path):
    """Every double is written as printf("%.15g"), which is what the
    reference's ostream at precision 15 produces."""
    case = cases.sod(40)
    cfg, mesh, fields = case
    rng = np.random.default_rng(3)
    vals = np.concatenate([[0.0, -0.0, 1.0, -1.5, 1e-300, 5e-324, 1.7976931348623157e308, np.inf, -np.inf,
                            0.1, 1 / 3, 123456789012345678.0, 2.5e-7, 1e15, 1e16, 999999999999999.5]],
                          axis=0)
    vals = np.concatenate([vals, rng.standard_normal(40 - vals.size) * 10.0 ** rng.integers(-20, 20, 40 - vals.size)])
    f = {k: v.copy() for k, v in fields.items()}
    g = cfg.nGhost
    f[abi.F_PRES][0, 0, g:-g] = vals
    vtk = abi.VtkSession(backends.cuda(), str(tmp_path), "fmt", cfg, mesh)
    vtk.write_host(0.25, f)
    vtk.close()
    text = (tmp_path / "snapshot_0" / "fmt_0_r0.vtr").read_text()
    block = text.split('Name="Pressure" format="ascii">\n', 1)[1].split("\n", 1)[0]
    assert block == "         " + "".join(" %.15g" % v for v in vals)
    pvd = (tmp_path / "fmt.pvd").read_text()
    assert '<DataSet timestep="0.25" file="snapshot_0/fmt_0.pvtr"/>' in pvd


def _nan_rule(ctx, cfg):
    """The reference's scan order restated in numpy."""
    names = [abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_PRES]
    if cfg.dim >= 2:
        names.append(abi.F_RHOV)
    if cfg.dim >= 3:
        names.append(abi.F_RHOW)
    arrs = [ctx.interior(ctx.get_field(f)).reshape(-1) for f in names]
    for cell in range(arrs[0].size):
        for f, a in zip(names, arrs):
            if np.isnan(a[cell]):
                return f, cell
    return -1, -1


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_oracle_nan_check(dim):
    case = {1: cases.sod(30), 2: cases.riemann2d(12), 3: cases.acoustic3d(5, semi=False, igr=False)}[dim]
    co = backends.make(backends.oracle(), case)
    assert co.check_nan() == (-1, -1)
    rng = np.random.default_rng(dim)
    fids = [abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_PRES] + ([abi.F_RHOV] if dim >= 2 else []) + \
        ([abi.F_RHOW] if dim >= 3 else [])
    for trial in range(6):
        c2 = backends.make(backends.oracle(), case)
        for _ in range(3):
            fid = fids[rng.integers(len(fids))]
            a = c2.get_field(fid)
            inner = c2.interior(a)
            idx = tuple(rng.integers(s) for s in inner.shape)
            inner[idx] = np.nan
            c2.set_field(fid, a)
        assert c2.check_nan() == _nan_rule(c2, case[0])
