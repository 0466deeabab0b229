"""Parity at the full sizes the benchmark runs.

The other parity tests run reduced grids; these run the benchmark's own
sizes, where index arithmetic, ragged tiles and long sweeps are exercised at
scale:

- 2D four-quadrant Riemann problem 4096 x 4096 (WENO5 + HLLC, SSP-RK3,
  CFL 0.6, outflow), reference-ordered FP64 on the GPU against the
  reference's own solver built from its sources (the C oracle where that
  build is absent), 2 steps: bit-identical fields and time steps.
- the same problem, fast FP64 against reference-ordered FP64 on the GPU for
  100 steps: relative L-infinity per conserved variable <= 1e-10.
- 3D acoustic pulse 256^3 periodic, semi-implicit RK1 + IGR + Jacobi,
  steps 0 and 1 (step 0 runs the 50-sweep IGR warm start) against the
  oracle: bit-identical fields, equal Jacobi iteration counts.

The CPU side takes about a minute per 2D step and per 3D step."""
import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-10   # relative L-infinity per conserved variable

FIELDS_2D = (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE, abi.F_VELU, abi.F_VELV, abi.F_PRES)
FIELDS_3D = (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOW, abi.F_RHOE, abi.F_VELU, abi.F_VELV, abi.F_VELW,
             abi.F_PRES, abi.F_SIGMA)


def _bitwise(cg, cc, fids):
    for fid in fids:
        a, b = cg.get_field(fid), cc.get_field(fid)
        ia, ib = cg.interior(a), cc.interior(b)
        rel = np.abs(ia - ib).max() / max(np.abs(ib).max(), 1e-300)
        assert rel <= TOL, f"field {fid}: relative L-inf {rel:.3e}"
        assert np.array_equal(ia.view(np.int64), ib.view(np.int64)), f"field {fid} differs (rel {rel:.3e})"


def test_riemann2d_4096_reference_order_bitwise():
    checker = backends.reference() or backends.oracle()
    case = cases.riemann2d(4096)
    case[0].precision = abi.PREC_FP64
    cg = backends.make(backends.cuda(), case)
    _, _, dtg = cases.run_steps(cg, 2)
    cc = backends.make(checker, cases.riemann2d(4096))
    _, _, dtc = cases.run_steps(cc, 2)
    assert dtg == dtc, (dtg, dtc)
    _bitwise(cg, cc, FIELDS_2D)
    print(f"4096^2 x 2 steps: CUDA reference order == {checker.name}, dt = {dtg}")


def test_riemann2d_4096_fast_fp64_within_tolerance_100_steps():
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_FP64_FAST):
        case = cases.riemann2d(4096)
        case[0].precision = prec
        c = backends.make(backends.cuda(), case)
        t, steps = c.advance(0, 0.0, -1.0, 100)
        assert steps == 100
        out[prec] = (t, {fid: c.interior(c.get_field(fid)).copy() for fid in FIELDS_2D[:4]})
        c.close()
    (te, ref), (tf, fast) = out[abi.PREC_FP64], out[abi.PREC_FP64_FAST]
    assert abs(tf - te) <= 1e-12 * te, (tf, te)
    worst = {}
    for fid, b in ref.items():
        worst[fid] = float(np.abs(fast[fid] - b).max() / np.abs(b).max())
    print("4096^2 x 100 steps, fast FP64 vs reference-ordered FP64, relative L-inf:", worst)
    assert max(worst.values()) <= TOL, worst


def test_acoustic3d_256_semi_implicit_steps_0_1_bitwise():
    case = cases.acoustic3d(256)
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), cases.acoustic3d(256))
    t = 0.0
    for step in (0, 1):
        dtg = cg.step(step, t, -1.0)
        dto = co.step(step, t, -1.0)
        assert dtg == dto, (step, dtg, dto)
        assert cg.last_pressure_iterations() == co.last_pressure_iterations(), step
        t += dtg
    _bitwise(cg, co, FIELDS_3D)
    print(f"256^3 semi-implicit steps 0-1: CUDA == oracle, Jacobi iterations {co.last_pressure_iterations()}")
