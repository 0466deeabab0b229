"""Pin the C oracle against the reference itself: the unmodified reference
sources compiled in place (oracle/_ref/libsifv_ref.so, -ffp-contract=off).

Every field (ghosts included) must be bit-identical after several steps,
over reconstruction orders, Riemann solvers, boundary conditions, EOS
kinds, multi-phase, IGR, and the semi-implicit Jacobi path."""
import ctypes

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

REF = backends.reference()
pytestmark = pytest.mark.skipif(REF is None, reason="reference build (oracle/_ref) not available")


def _fields(cfg):
    f = [abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_VELU, abi.F_PRES, abi.F_SIGMA]
    if cfg.dim >= 2:
        f += [abi.F_RHOV, abi.F_VELV]
    if cfg.dim >= 3:
        f += [abi.F_RHOW, abi.F_VELW]
    for p in range(cfg.nPhases):
        f += [abi.F_ALPHARHO(p), abi.F_ALPHA(p)]
    return f


def _compare(case, nsteps, t_end=None):
    co = backends.make(backends.oracle(), case)
    cr = backends.make(REF, case)
    _, _, dto = cases.run_steps(co, nsteps, t_end)
    _, _, dtr = cases.run_steps(cr, nsteps, t_end)
    assert dto == dtr
    for fid in _fields(case[0]):
        a, b = co.get_field(fid), cr.get_field(fid)
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), f"field {fid} differs (max {np.abs(a - b).max()})"
    if case[0].semiImplicit:
        assert co.last_pressure_iterations() == cr.last_pressure_iterations()


@pytest.mark.parametrize("recon", [abi.WENO1, abi.WENO3, abi.WENO5, abi.UPWIND1, abi.UPWIND3, abi.UPWIND5])
@pytest.mark.parametrize("riemann", [abi.LF, abi.RUSANOV, abi.HLLC])
def test_sod_orders_and_solvers(recon, riemann):
    _compare(cases.sod(120, recon=recon, riemann=riemann), 40)


@pytest.mark.parametrize("bc", [abi.BC_OUTFLOW, abi.BC_PERIODIC, abi.BC_SLIPWALL, abi.BC_NOSLIPWALL, abi.BC_SYMMETRY])
def test_riemann2d_boundaries(bc):
    _compare(cases.riemann2d(20, bc=bc), 6)


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_water_air_multiphase(rk):
    _compare(cases.water_air(96, rk=rk), 25)


@pytest.mark.parametrize("riemann", [abi.HLLC, abi.RUSANOV, abi.LF])
def test_water_air_solvers(riemann):
    _compare(cases.water_air(64, riemann=riemann), 15)


@pytest.mark.parametrize("rk,igr", [(1, True), (3, True), (2, False)])
def test_acoustic3d_semi_implicit(rk, igr):
    _compare(cases.acoustic3d(8, rk=rk, igr=igr), 3)


def test_explicit_3d_igr_lf():
    case = cases.acoustic3d(8, semi=False, igr=True, rk=3, riemann=abi.LF)
    case[0].cfl = 0.5
    _compare(case, 3)


def test_stiffened_single_phase():
    case = cases.sod(80)
    case[0].eosKind = abi.EOS_STIFFENED
    case[0].pInf = 0.5
    _compare(case, 20)


def test_body_force():
    case = cases.riemann2d(16, rk=2)
    for d, (a, b, c) in enumerate([(0.1, 0.05, 3.0), (-0.2, 0.0, 0.0)]):
        case[0].bfA[d], case[0].bfB[d], case[0].bfC[d] = a, b, c
    _compare(case, 5)


def test_semi_implicit_multiphase():
    case = cases.water_air(48, p_left=2e5, rk=1)
    case[0].semiImplicit = 1
    case[0].siCfl = 0.5
    case[0].siMaxDt = 1e-5
    _compare(case, 4)


def test_gauss_seidel_pressure_solver():
    case = cases.advection1d(64, semi=True)
    co = backends.make(backends.oracle(), case)
    cr = backends.make(REF, case)
    co.set_pressure_solver(1)
    cr.set_pressure_solver(1)
    cases.run_steps(co, 5)
    cases.run_steps(cr, 5)
    for fid in _fields(case[0]):
        assert np.array_equal(co.get_field(fid), cr.get_field(fid))


def test_standalone_pressure_solve_and_dt():
    case = cases.acoustic3d(8)
    co = backends.make(backends.oracle(), case)
    cr = backends.make(REF, case)
    rng = np.random.default_rng(7)
    n = co.ncells
    rho = 1.0 + 0.1 * rng.random(n)
    rhoc2 = 1.4 + 0.2 * rng.random(n)
    rhs = rng.random(n)
    p0 = rng.random(n)
    po, io, _ = co.pressure_solve(rho, rhoc2, rhs, p0, 1e-2, 1e-10, 50)
    pr, ir, _ = cr.pressure_solve(rho, rhoc2, rhs, p0, 1e-2, 1e-10, 50)
    assert io == ir
    assert np.array_equal(co.interior(po), cr.interior(pr))
    assert co.acoustic_dt(0.6, 1.0) == cr.acoustic_dt(0.6, 1.0)
    assert co.advective_dt(0.8, 1.0) == cr.advective_dt(0.8, 1.0)


@pytest.mark.parametrize("name", cases.VISCOUS_CASES)
def test_viscous_stress(name):
    """addViscousFluxes (src/ViscousFlux.cpp) and computeViscousDt
    (src/RKTimeStepping.cpp:161-188) in the explicit and semi-implicit steps."""
    case, n = cases.viscous(name)
    _compare(case, n)


def test_viscous_config_validation():
    lib = backends.oracle()
    bad = abi.config_defaults(dim=1, nGhost=3, reconOrder=abi.WENO5)
    bad.mu = -1.0
    assert lib.fn["config_validate"](ctypes.byref(bad)) == abi.ERR_BAD_CONFIG
    bad.mu, bad.nPhaseMu = 0.0, 2
    assert lib.fn["config_validate"](ctypes.byref(bad)) == abi.ERR_BAD_CONFIG


def test_viscous_3d_explicit_walls():
    """All three face directions, transverse gradients through corner ghosts
    of mixed wall kinds, RK2 + LF."""
    case = cases.acoustic3d(9, semi=False, igr=False, rk=2, riemann=abi.LF)
    case[0].mu = 0.03
    case[1].bc = [abi.BC_NOSLIPWALL, abi.BC_SLIPWALL, abi.BC_NOSLIPWALL, abi.BC_OUTFLOW,
                  abi.BC_SYMMETRY, abi.BC_NOSLIPWALL]
    _compare(case, 4)


@pytest.mark.parametrize("name", cases.CAPILLARY_CASES)
def test_surface_tension(name):
    """addSurfaceTensionFluxes (src/SurfaceTension.cpp) and computeCapillaryDt
    (src/RKTimeStepping.cpp:201-228), explicit and semi-implicit, 2D and 3D,
    alone and after the viscous stress."""
    case, n = cases.capillary(name)
    _compare(case, n)


def test_surface_tension_config_validation():
    lib = backends.oracle()
    bad = abi.config_defaults(dim=2, nGhost=3, reconOrder=abi.WENO5, nPhases=2, phaseGamma=[4.4, 1.4],
                              phasePInf=[6e8, 0.0])
    bad.stSigma = -1.0
    assert lib.fn["config_validate"](ctypes.byref(bad)) == abi.ERR_BAD_CONFIG
    bad.stSigma, bad.stEpsGradAlpha = 0.07, 0.0
    assert lib.fn["config_validate"](ctypes.byref(bad)) == abi.ERR_BAD_CONFIG
    bad.stEpsGradAlpha = 1e-8
    assert lib.fn["config_validate"](ctypes.byref(bad)) == abi.OK
    bad.nPhases = 0
    assert lib.fn["config_validate"](ctypes.byref(bad)) == abi.ERR_BAD_CONFIG


@pytest.mark.parametrize("name", cases.IB_CASES)
def test_immersed_boundary(name):
    """ImmersedBoundaryMethod (src/ImmersedBoundary.cpp): classifyCells with
    the four body shapes, applyGhostCells per stage, solid cells out of the
    update, the dt limit and the IGR sweeps."""
    case, bodies, n = cases.immersed(name)
    ref = backends.reference()
    cr = backends.make(ref, case)
    co = backends.make(backends.oracle(), case)
    cr.set_immersed_bodies(bodies)
    co.set_immersed_bodies(bodies)
    types = co.ib_cell_types()
    assert np.array_equal(types, cr.ib_cell_types())
    assert (types == abi.CELL_GHOST).sum() > 0 and (types == abi.CELL_DEAD).sum() > 0
    _, _, dr = cases.run_steps(cr, n)
    _, _, do = cases.run_steps(co, n)
    assert dr == do
    for fid in cases.output_fields(co, case[0]):
        assert np.array_equal(co.get_field(fid), cr.get_field(fid)), fid
