"""Mixed-precision semi-implicit step (SIFV_PREC_MIXED with semiImplicit):
the Jacobi pressure solve runs FP32 inner sweeps inside FP64 iterative
refinement, everything else stays the reference-ordered FP64 step.  The
solve must stop at the reference's iteration (max change < tol, to FP32
rounding of the change) and the step must stay within the pressure
tolerance of the FP64 oracle."""
import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["acoustic3d", "box2d_walls", "advection1d"])
def test_mixed_semi_step_within_tolerance_of_fp64(name):
    if name == "acoustic3d":
        case = cases.acoustic3d(16)
    elif name == "box2d_walls":
        case = cases.acoustic_box(48, 40, bc=abi.BC_SLIPWALL, stretch=0.02, tol=1e-7)
    else:
        case = cases.advection1d(96, semi=True)
    tol = case[0].pressureTol
    co = backends.make(backends.oracle(), case)
    case[0].precision = abi.PREC_MIXED
    cm = backends.make(backends.cuda(), case)
    for s in range(4):
        t = 0.0
        dm = cm.step(s, t)
        do = co.step(s, t)
        assert dm == do if s == 0 else abs(dm - do) <= 1e-6 * do
        im, io = cm.last_pressure_iterations(), co.last_pressure_iterations()
        assert abs(im - io) <= 1, (s, im, io)
    for fid in (abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_PRES):
        a, b = cm.interior(cm.get_field(fid)), co.interior(co.get_field(fid))
        scale = np.abs(b).max()
        err = np.abs(a - b).max()
        assert err <= 20 * tol * max(scale, 1.0), (fid, err)


def test_mixed_standalone_solve_matches_fp64_iterations():
    case = cases.acoustic3d(12)
    case[0].precision = abi.PREC_MIXED
    cm = backends.make(backends.cuda(), case)
    case[0].precision = abi.PREC_FP64
    cg = backends.make(backends.cuda(), case)
    rng = np.random.default_rng(4)
    n = cg.ncells
    args = (1.0 + 0.1 * rng.random(n), 1.4 + 0.2 * rng.random(n), rng.random(n), rng.random(n))
    for tol in (1e-6, 1e-9):
        pm, im, _ = cm.pressure_solve(*args, 0.1, tol, 2000)
        pg, ig, _ = cg.pressure_solve(*args, 0.1, tol, 2000)
        assert abs(im - ig) <= 1, (tol, im, ig)
        assert np.abs(cm.interior(pm) - cg.interior(pg)).max() <= 10 * tol


def test_fast_precision_still_rejects_semi_implicit():
    case = cases.acoustic3d(8)
    case[0].precision = abi.PREC_FP64_FAST
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(case[0], case[1])
    assert e.value.status == abi.ERR_UNSUPPORTED
