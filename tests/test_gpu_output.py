"""runTimeLoop on the GPU (sifv_run_time_loop) with VTK output from the
device state (sifv_vtk_write) and the device NaN check (sifv_check_nan):

- files byte-identical to the reference's own runTimeLoop + VTKSession and
  the final state bit-identical, on the device-resident loop (explicit) and
  the host-driven one (IGR / semi-implicit), for several batch sizes;
- the NaN check against the oracle's, and the loop stopping at the first
  output that holds a NaN;
- snapshots taken while the context keeps stepping hold the state of the
  moment they were requested."""
import filecmp
import os

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu


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
    if name == "sod":
        case = cases.sod(64)
    elif name == "riemann2d":
        case = cases.riemann2d(20, bc=abi.BC_SLIPWALL)
    elif name == "water_air":
        case = cases.water_air(48)
    elif name == "acoustic3d_igr":
        case = cases.acoustic3d(6)
    elif name == "acoustic3d_semi_noigr":
        case = cases.acoustic3d(6, igr=False)
    elif name == "droplet2d":
        case = cases.droplet(16)
    else:
        raise KeyError(name)
    probe = backends.make(backends.oracle(), case)
    dt0 = probe.step(0, 0.0, -1.0)
    return case, 5.5 * dt0, 2.2 * dt0


@pytest.mark.parametrize("name,batch", [("sod", 0), ("sod", 1), ("riemann2d", 3), ("water_air", 2),
                                        ("acoustic3d_igr", 0), ("acoustic3d_semi_noigr", 0), ("droplet2d", 4)])
def test_time_loop_matches_reference(name, batch, tmp_path):
    ref = backends.reference()
    if ref is None:
        pytest.skip("reference library not built")
    case, t_end, every = loop_case(name)
    cr = backends.make(ref, case)
    steps_ref = cr.reference_time_loop(str(tmp_path / "ref"), name, t_end, every)

    cg = backends.make(backends.cuda(), case)
    vtk = abi.VtkSession(backends.cuda(), str(tmp_path / "gpu"), name, case[0], case[1])
    seen = []
    st, r = cg.run_time_loop(t_end, every, vtk=vtk, batch=batch, progress=lambda s, t, dt: seen.append((s, t, dt)))
    vtk.close()
    assert st == abi.OK
    assert r.steps == steps_ref and r.nanField == -1
    assert_same_tree(str(tmp_path / "ref"), str(tmp_path / "gpu"))
    for fid in cases.output_fields(cg, case[0]):
        assert np.array_equal(cg.get_field(fid), cr.get_field(fid)), fid

    co = backends.make(backends.oracle(), case)
    printed = []
    t, n = cases.run_time_loop(co, t_end, every, print_interval=1, on_print=lambda s, tt, dt: printed.append((s, tt, dt)))
    assert printed == seen and r.time == t


def test_time_loop_fast_path_matches_stepping():
    """The device-resident loop over the fused 2D stage kernel takes the
    same steps as sifv_step driven by the reference's loop."""
    case = cases.riemann2d(96)
    case[0].precision = abi.PREC_FP64_FAST
    c1 = backends.make(backends.cuda(), case)
    c2 = backends.make(backends.cuda(), case)
    t1, n1 = cases.run_time_loop(c1, 0.05, 0.012)
    st, r = c2.run_time_loop(0.05, 0.012, batch=5)
    assert st == abi.OK and r.steps == n1 and r.time == t1 and r.outputs == 5
    for fid in (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE, abi.F_PRES):
        assert np.array_equal(c1.get_field(fid), c2.get_field(fid)), fid


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_check_nan_matches_oracle(dim):
    case = {1: cases.sod(300), 2: cases.riemann2d(40), 3: cases.acoustic3d(12, semi=False, igr=False)}[dim]
    fids = [abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_PRES] + ([abi.F_RHOV] if dim >= 2 else []) + \
        ([abi.F_RHOW] if dim >= 3 else [])
    rng = np.random.default_rng(10 + dim)
    cg = backends.make(backends.cuda(), case)
    assert cg.check_nan() == (-1, -1)
    for trial in range(8):
        cg = backends.make(backends.cuda(), case)
        co = backends.make(backends.oracle(), case)
        for _ in range(1 + trial % 4):
            fid = fids[rng.integers(len(fids))]
            a = cg.get_field(fid)
            inner = cg.interior(a)
            inner[tuple(rng.integers(s) for s in inner.shape)] = np.nan
            cg.set_field(fid, a)
            co.set_field(fid, a)
        assert cg.check_nan() == co.check_nan()


def test_time_loop_stops_at_first_output_with_nan(tmp_path):
    case = cases.riemann2d(32)
    cfg, mesh, fields = case
    f = {k: v.copy() for k, v in fields.items()}
    g = cfg.nGhost
    f[abi.F_RHOE][0, g + 20, g + 7] = np.nan
    bad = (cfg, mesh, f)
    co = backends.make(backends.oracle(), bad)
    outs = []
    cases.run_time_loop(co, 0.05, 0.02, on_output=lambda t, s: outs.append((t, s)))
    cg = backends.make(backends.cuda(), bad)
    vtk = abi.VtkSession(backends.cuda(), str(tmp_path), "nan", cfg, mesh)
    st, r = cg.run_time_loop(0.05, 0.02, vtk=vtk)
    vtk.close()
    assert st == abi.ERR_NAN
    assert (r.nanTime, r.nanStep) == outs[1] and r.outputs == 2
    assert (r.nanField, r.nanCell) == cg.check_nan() and r.nanField >= 0
    assert sorted(os.listdir(tmp_path)) == ["nan.pvd", "snapshot_0", "snapshot_1"]


def test_device_snapshots_while_stepping(tmp_path):
    """Each sifv_vtk_write captures the state at the call, although the
    context steps on before the files are written."""
    case = cases.riemann2d(64)
    cfg, mesh, _ = case
    cg = backends.make(backends.cuda(), case)
    dev = abi.VtkSession(backends.cuda(), str(tmp_path / "dev"), "s", cfg, mesh)
    host = abi.VtkSession(backends.cuda(), str(tmp_path / "host"), "s", cfg, mesh)
    t = 0.0
    for n in range(5):
        dev.write(cg, t)
        host.write_host(t, cases.output_fields(cg, cfg))
        for k in range(3):
            t += cg.step(3 * n + k, t)
    dev.close()
    host.close()
    assert_same_tree(str(tmp_path / "dev"), str(tmp_path / "host"))
