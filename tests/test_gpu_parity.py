"""Parity of the CUDA library (through the C ABI) against the C oracle.

The FP64 build evaluates every expression in the reference's order without
FMA contraction, so the expected result is bit-identical fields; the
acceptance bar (relative L-infinity <= 1e-10 per variable, the pressure
solve to pressureTol) is asserted as well and reported separately."""
import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-10   # relative L-infinity per conserved variable


def _fields(cfg):
    f = [abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_VELU, abi.F_PRES, abi.F_SIGMA]
    if cfg.dim >= 2:
        f += [abi.F_RHOV, abi.F_VELV]
    if cfg.dim >= 3:
        f += [abi.F_RHOW, abi.F_VELW]
    for p in range(cfg.nPhases):
        f += [abi.F_ALPHARHO(p), abi.F_ALPHA(p)]
    return f


def run_pair(case, nsteps, t_end=None):
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    tg, sg, dtg = cases.run_steps(cg, nsteps, t_end)
    to, so, dto = cases.run_steps(co, nsteps, t_end)
    return cg, co, dtg, dto


def check(case, nsteps, t_end=None, bitwise=True):
    cg, co, dtg, dto = run_pair(case, nsteps, t_end)
    assert len(dtg) == len(dto)
    np.testing.assert_allclose(dtg, dto, rtol=TOL, atol=0)
    worst = {}
    for fid in _fields(case[0]):
        a, b = cg.get_field(fid), co.get_field(fid)
        ia, ib = cg.interior(a), co.interior(b)
        scale = max(np.abs(ib).max(), 1e-300)
        rel = np.abs(ia - ib).max() / scale
        worst[fid] = rel
        assert rel <= TOL, f"field {fid}: relative L-inf {rel:.3e} > {TOL}"
        if bitwise:
            assert np.array_equal(a.view(np.int64), b.view(np.int64)), \
                f"field {fid} not bit-identical (rel {rel:.3e})"
    if case[0].semiImplicit:
        assert cg.last_pressure_iterations() == co.last_pressure_iterations()
    return worst


def test_sod_full_config():
    """Config 1 in full: 1000 cells, WENO5 + HLLC, RK3, CFL 0.6, to t = 0.2."""
    check(cases.sod(1000), 100000, t_end=0.2)


@pytest.mark.parametrize("recon", [abi.WENO1, abi.WENO3, abi.WENO5, abi.UPWIND1, abi.UPWIND3, abi.UPWIND5])
@pytest.mark.parametrize("riemann", [abi.LF, abi.RUSANOV, abi.HLLC])
def test_sod_orders_solvers(recon, riemann):
    check(cases.sod(120, recon=recon, riemann=riemann), 30)


@pytest.mark.parametrize("bc", [abi.BC_OUTFLOW, abi.BC_PERIODIC, abi.BC_SLIPWALL, abi.BC_NOSLIPWALL,
                                abi.BC_SYMMETRY])
def test_riemann2d_boundaries(bc):
    check(cases.riemann2d(40, bc=bc), 8)


def test_riemann2d_many_steps():
    check(cases.riemann2d(96), 60)


def test_riemann2d_weno_eps_example():
    check(cases.riemann2d(64, weno_eps=1e-16), 20)


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_water_air(rk):
    check(cases.water_air(200, rk=rk), 40)


def test_water_air_config5_instance():
    check(cases.water_air(1024, x_interface=0.43, p_left=7.3e8), 300, t_end=1e-4)


@pytest.mark.parametrize("rk,igr", [(1, True), (3, True), (2, False)])
def test_acoustic3d_semi_implicit(rk, igr):
    check(cases.acoustic3d(16, rk=rk, igr=igr), 3)


@pytest.mark.parametrize("bc,stretch", [(abi.BC_PERIODIC, 0.0), (abi.BC_SLIPWALL, 0.02)])
def test_igr_tiled_wavefront_3d_ragged(bc, stretch):
    """Several 16^3 IGR tiles with ragged edges (40 x 36 x 20 cells)."""
    check(cases.acoustic_box(40, 36, 20, bc=bc, stretch=stretch), 2)


@pytest.mark.parametrize("nx,ny,nz", [(48, 34, 40), (35, 40, 33)])
def test_igr_record_sweep_3d(nx, ny, nz):
    """3D IGR sweeps with precomputed reciprocals (even row length: 48 + 6
    ghosts, tiles ragged in y and z) and the plain tile sweep they fall back to
    (odd row length: 35 + 6 ghosts), both bit-identical to the oracle."""
    check(cases.acoustic_box(nx, ny, nz, bc=abi.BC_SLIPWALL, stretch=0.01), 2)


@pytest.mark.parametrize("shape,bcs", [((40, 36, 34), (abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_SLIPWALL)),
                                        ((34, 20, 50), (abi.BC_OUTFLOW, abi.BC_SYMMETRY, abi.BC_PERIODIC)),
                                        ((50, 40, 18), (abi.BC_PERIODIC, abi.BC_PERIODIC, abi.BC_NOSLIPWALL)),
                                        ((35, 40, 33), (abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_PERIODIC)),
                                        ((100, 140, 1), (abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_OUTFLOW)),
                                        ((130, 70, 1), (abi.BC_SLIPWALL, abi.BC_PERIODIC, abi.BC_OUTFLOW)),
                                        ((208, 64, 48), (abi.BC_SLIPWALL, abi.BC_OUTFLOW, abi.BC_OUTFLOW)),
                                        ((600, 520, 1), (abi.BC_OUTFLOW, abi.BC_SLIPWALL, abi.BC_OUTFLOW)),
                                        ((90, 159, 1), (abi.BC_PERIODIC, abi.BC_PERIODIC, abi.BC_OUTFLOW))])
@pytest.mark.parametrize("march", [True, False])
def test_igr_overlapped_sweeps_mixed_faces(shape, bcs, march, monkeypatch):
    """Consecutive sweeps overlapped in one launch sequence (sweep s + 1
    trailing sweep s by a fixed number of tile planes, boundary tiles
    refreshing the ghost layer themselves) -- the 3D record sweep, the plain
    3D tile sweep of odd row lengths (35 + 6 ghosts) and the 2D 32 x 64 tile
    sweep -- with per-axis boundary kinds (periodic wrap images and
    zero-gradient copies), several tiles along the periodic axes, ragged
    edges, more than eight sweeps in one launch (18 and 27 tile planes at a
    lag of 2), the 20-sweep warm start: bit-identical to the oracle's
    sweep-by-sweep order.  2D meshes run both 2D paths: the persistent
    wavefront (SIFV_GS_MARCH=1) and the tiled sweeps (SIFV_GS_MARCH=0)."""
    if shape[2] > 1 and not march:
        pytest.skip("3D meshes have one path")
    monkeypatch.setenv("SIFV_GS_MARCH", "1" if march else "0")
    cfg, mesh, fields = cases.acoustic_box(*shape)
    mesh.bc = [bcs[0]] * 2 + [bcs[1]] * 2 + [bcs[2]] * 2
    check((cfg, mesh, fields), 2)


@pytest.mark.parametrize("bc", [abi.BC_PERIODIC, abi.BC_OUTFLOW])
def test_igr_tiled_wavefront_2d_ragged(bc):
    """Several 32 x 64 IGR tiles with ragged edges (100 x 140 cells)."""
    check(cases.acoustic_box(100, 140, bc=bc, stretch=0.01), 2)


def test_explicit_3d_igr_lf():
    case = cases.acoustic3d(12, semi=False, igr=True, rk=3, riemann=abi.LF)
    case[0].cfl = 0.5
    check(case, 3)


def test_stiffened_and_body_force():
    case = cases.riemann2d(32, rk=2)
    case[0].eosKind = abi.EOS_STIFFENED
    case[0].pInf = 0.3
    case[0].bfA[0], case[0].bfB[0], case[0].bfC[0] = 0.1, 0.05, 3.0
    case[0].bfA[1] = -0.2
    check(case, 6)


def test_semi_implicit_multiphase():
    case = cases.water_air(64, p_left=2e5, rk=1)
    case[0].semiImplicit = 1
    case[0].siCfl = 0.5
    case[0].siMaxDt = 1e-5
    check(case, 4)


def test_standalone_pressure_solve_dt_and_igr():
    case = cases.acoustic3d(12)
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    rng = np.random.default_rng(11)
    n = cg.ncells
    rho = 1.0 + 0.1 * rng.random(n)
    rhoc2 = 1.4 + 0.2 * rng.random(n)
    rhs = rng.random(n)
    p0 = rng.random(n)
    pg, ig, _ = cg.pressure_solve(rho, rhoc2, rhs, p0, 1e-2, 1e-12, 60)
    po, io, _ = co.pressure_solve(rho, rhoc2, rhs, p0, 1e-2, 1e-12, 60)
    assert ig == io
    assert np.array_equal(cg.interior(pg), co.interior(po))
    assert cg.acoustic_dt(0.6, 1.0) == co.acoustic_dt(0.6, 1.0)
    assert cg.advective_dt(0.8, 1.0) == co.advective_dt(0.8, 1.0)
    for c in (cg, co):
        c.convert_cons_to_prim()
        c.apply_bc()
        c.igr_solve(0)
    assert np.array_equal(cg.get_field(abi.F_SIGMA), co.get_field(abi.F_SIGMA))


@pytest.mark.parametrize("bc", [abi.BC_PERIODIC, abi.BC_SLIPWALL, abi.BC_OUTFLOW])
@pytest.mark.parametrize("max_iter,dt,tol", [(7, 2e-3, 1e-14), (8, 2e-3, 1e-14), (200, 2e-3, 1e-8),
                                             (200, 1e-2, 1e-8), (200, 1e-2, 1e-7)])
def test_jacobi_3d_uniform_axes(bc, max_iter, dt, tol):
    """3D Jacobi on axes of equal cell widths (per-face coefficients,
    k_jacobi3<true>, ragged 32 x 8 column tiles and 16-cell z segments):
    iteration counts -- odd and even caps, convergence after an odd or an
    even number of iterations, several host batches -- and the iterate are
    the oracle's bit for bit."""
    cfg, mesh, fields = cases.acoustic_box(40, 20, 37, bc=bc)
    mesh.x, mesh.y, mesh.z = np.arange(41) / 64.0, np.arange(21) / 64.0, np.arange(38) / 64.0   # equal widths
    cg = backends.make(backends.cuda(), (cfg, mesh, fields))
    co = backends.make(backends.oracle(), (cfg, mesh, fields))
    rng = np.random.default_rng(max_iter + bc)
    n = cg.ncells
    args = (1.0 + 0.1 * rng.random(n), 1.4 + 0.2 * rng.random(n), rng.random(n), rng.random(n))
    pg, ig, _ = cg.pressure_solve(*args, dt, tol, max_iter)
    po, io, _ = co.pressure_solve(*args, dt, tol, max_iter)
    assert ig == io, (ig, io)
    assert np.array_equal(cg.interior(pg), co.interior(po))


@pytest.mark.parametrize("plant", ["sigma", "rho"])
def test_igr_record_sweep_fallbacks(plant):
    """The record sweep's exact-quotient guards: planted -0, tiny and huge
    sigma values send those cells to plain divisions; densities of 1e200 put
    face reciprocals outside the fast range, so the whole solve divides
    plainly.  Either way sigma stays bit-identical to the oracle's sweeps."""
    case = cases.acoustic_box(48, 34, 40, bc=abi.BC_PERIODIC)
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    for c in (cg, co):
        c.convert_cons_to_prim()
        c.apply_bc()
    if plant == "sigma":
        sig = cg.get_field(abi.F_SIGMA)
        flat = sig.reshape(-1)
        rng = np.random.default_rng(5)
        flat[:] = 1e-3 * rng.random(flat.size)
        idx = rng.choice(flat.size, 400, replace=False)
        flat[idx[0::4]] = -0.0
        flat[idx[1::4]] = 1e-200
        flat[idx[2::4]] = -1e200
        flat[idx[3::4]] = 0.0
        for c in (cg, co):
            c.set_field(abi.F_SIGMA, sig)
    else:
        rho = cg.get_field(abi.F_RHO)
        inner = cg.interior(rho)
        inner[::7, ::5, ::9] = 1e200
        for c in (cg, co):
            c.set_field(abi.F_RHO, rho)
            c.apply_bc()
    for c in (cg, co):
        c.igr_solve(1)
    a, b = cg.get_field(abi.F_SIGMA), co.get_field(abi.F_SIGMA)
    assert np.array_equal(a.view(np.int64), b.view(np.int64))


def test_not_converged_status():
    case = cases.acoustic3d(8)
    cg = backends.make(backends.cuda(), case)
    n = cg.ncells
    _, iters, st = cg.pressure_solve(np.ones(n), np.ones(n), np.ones(n), np.zeros(n), 1.0, 1e-30, 1)
    assert iters == 1 and st == abi.NOT_CONVERGED


def test_bad_config_rejected():
    cfg, mesh, _ = cases.sod(50)
    cfg.nGhost = 1
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(cfg, mesh)
    assert e.value.status == abi.ERR_BAD_CONFIG


def test_advance_matches_step():
    case = cases.riemann2d(48)
    c1 = backends.make(backends.cuda(), case)
    c2 = backends.make(backends.cuda(), case)
    t1, s1, _ = cases.run_steps(c1, 7, t_end=0.05)
    t2, s2 = c2.advance(0, 0.0, 0.05, 7)
    assert s1 == s2 and t1 == t2
    for fid in (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE, abi.F_PRES):
        assert np.array_equal(c1.get_field(fid), c2.get_field(fid))


def _check_with_solver(case, nsteps, kind):
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    cg.set_pressure_solver(kind)
    co.set_pressure_solver(kind)
    _, _, dtg = cases.run_steps(cg, nsteps)
    _, _, dto = cases.run_steps(co, nsteps)
    assert dtg == dto
    for fid in _fields(case[0]):
        a, b = cg.get_field(fid), co.get_field(fid)
        assert np.array_equal(cg.interior(a), co.interior(b)), fid
    assert cg.last_pressure_iterations() == co.last_pressure_iterations()
    return cg.last_pressure_iterations()


@pytest.mark.parametrize("shape,bcs,segs", [((100, 140, 1), (abi.BC_OUTFLOW, abi.BC_SLIPWALL), 2),
                                            ((130, 70, 1), (abi.BC_SLIPWALL, abi.BC_OUTFLOW), 3),
                                            ((600, 520, 1), (abi.BC_OUTFLOW, abi.BC_SLIPWALL), 5),
                                            ((90, 159, 1), (abi.BC_SYMMETRY, abi.BC_OUTFLOW), 0)])
@pytest.mark.parametrize("max_iter,dt,tol", [(2, 1e-2, 1e-14), (7, 1e-2, 1e-14), (300, 2e-3, 1e-9)])
def test_gauss_seidel_wavefront_segments(shape, bcs, segs, max_iter, dt, tol, monkeypatch):
    """The 2D wavefront on meshes without a periodic face, rows cut into
    segments along the march axis (SIFV_GS_MARCH_SEGMENTS; 0 = the count
    the solver picks): iteration count and the whole returned array are
    the oracle's bit for bit."""
    monkeypatch.setenv("SIFV_GS_MARCH", "1")
    monkeypatch.setenv("SIFV_GS_MARCH_SEGMENTS", str(segs))
    cfg, mesh, fields = cases.acoustic_box(*shape)
    mesh.bc = [bcs[0]] * 2 + [bcs[1]] * 2 + [abi.BC_OUTFLOW] * 2
    cg = backends.make(backends.cuda(), (cfg, mesh, fields))
    co = backends.make(backends.oracle(), (cfg, mesh, fields))
    cg.set_pressure_solver(abi.PRESSURE_GAUSS_SEIDEL)
    co.set_pressure_solver(abi.PRESSURE_GAUSS_SEIDEL)
    rng = np.random.default_rng(max_iter + segs)
    n = cg.ncells
    args = (1.0 + 0.1 * rng.random(n), 1.4 + 0.2 * rng.random(n), rng.random(n), rng.random(n))
    pg, ig, _ = cg.pressure_solve(*args, dt, tol, max_iter)
    po, io, _ = co.pressure_solve(*args, dt, tol, max_iter)
    assert ig == io, (ig, io)
    assert np.array_equal(pg.view(np.int64), po.view(np.int64))


@pytest.mark.parametrize("shape,bcs,segs", [((100, 140, 1), (abi.BC_OUTFLOW, abi.BC_SLIPWALL), 3),
                                            ((600, 520, 1), (abi.BC_SLIPWALL, abi.BC_OUTFLOW), 4)])
def test_igr_wavefront_segments(shape, bcs, segs, monkeypatch):
    """IGR sweeps (20-sweep warm start, then 5) in the 2D wavefront with
    rows cut into segments, through two steps: bit-identical to the oracle."""
    monkeypatch.setenv("SIFV_GS_MARCH", "1")
    monkeypatch.setenv("SIFV_GS_MARCH_SEGMENTS", str(segs))
    cfg, mesh, fields = cases.acoustic_box(*shape)
    mesh.bc = [bcs[0]] * 2 + [bcs[1]] * 2 + [abi.BC_OUTFLOW] * 2
    check((cfg, mesh, fields), 2)


@pytest.mark.parametrize("bcs", [(abi.BC_PERIODIC, abi.BC_PERIODIC), (abi.BC_PERIODIC, abi.BC_SLIPWALL),
                                 (abi.BC_OUTFLOW, abi.BC_PERIODIC)])
def test_semi_implicit_2d_periodic_wavefront_steps(bcs):
    """Three semi-implicit steps on 2D meshes with a periodic face (IGR warm
    start and 5-sweep solves, Gauss-Seidel pressure solves to tol 1e-8): both
    run as the persistent wavefront, walking along x (periodic x), along y
    (periodic y only) or along the longer axis (both periodic, 200 x 300);
    several CTAs of 32-row groups.  Every field, dt and the iteration counts
    are the oracle's bit for bit."""
    nx, ny = (200, 300) if bcs == (abi.BC_PERIODIC, abi.BC_PERIODIC) else (300, 200)
    cfg, mesh, fields = cases.acoustic_box(nx, ny)
    mesh.bc = [bcs[0]] * 2 + [bcs[1]] * 2 + [abi.BC_OUTFLOW] * 2
    iters = _check_with_solver((cfg, mesh, fields), 3, 1)
    assert iters > 1


@pytest.mark.parametrize("name", ["advection1d", "acoustic3d", "box3d_ragged", "box2d_ragged"])
def test_gauss_seidel_pressure_solver(name):
    """GaussSeidelPressureSolver as the semi-implicit step's plugin: tiled
    wavefront sweeps bit-identical to the lexicographic in-place order."""
    if name == "advection1d":
        case = cases.advection1d(64, semi=True)
        case[0].pressureTol = 1e-13
    elif name == "acoustic3d":
        case = cases.acoustic3d(16)
    elif name == "box3d_ragged":
        case = cases.acoustic_box(40, 36, 20, bc=abi.BC_SLIPWALL, stretch=0.02)
    else:
        case = cases.acoustic_box(100, 140, bc=abi.BC_PERIODIC)
    iters = _check_with_solver(case, 3, 1)
    assert iters > 1


@pytest.mark.parametrize("shape,bcs", [((40, 36, 34), (abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_SLIPWALL)),
                                        ((34, 20, 50), (abi.BC_OUTFLOW, abi.BC_SYMMETRY, abi.BC_PERIODIC)),
                                        ((50, 40, 18), (abi.BC_PERIODIC, abi.BC_PERIODIC, abi.BC_NOSLIPWALL)),
                                        ((64, 32, 32), (abi.BC_PERIODIC, abi.BC_PERIODIC, abi.BC_PERIODIC)),
                                        ((35, 40, 33), (abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_PERIODIC)),
                                        ((100, 140, 1), (abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_OUTFLOW)),
                                        ((130, 70, 1), (abi.BC_SLIPWALL, abi.BC_PERIODIC, abi.BC_OUTFLOW)),
                                        ((600, 520, 1), (abi.BC_OUTFLOW, abi.BC_SLIPWALL, abi.BC_OUTFLOW)),
                                        ((330, 200, 1), (abi.BC_OUTFLOW, abi.BC_PERIODIC, abi.BC_OUTFLOW)),
                                        ((90, 159, 1), (abi.BC_PERIODIC, abi.BC_PERIODIC, abi.BC_OUTFLOW))])
@pytest.mark.parametrize("max_iter,dt,tol", [(1, 1e-2, 1e-14), (2, 1e-2, 1e-14), (3, 1e-2, 1e-14),
                                             (7, 1e-2, 1e-14), (300, 2e-3, 1e-9), (300, 1e-2, 1e-8)])
@pytest.mark.parametrize("march", [True, False])
def test_gauss_seidel_overlapped_iterations(shape, bcs, max_iter, dt, tol, march, monkeypatch):
    """Gauss-Seidel iterations overlapped in one launch sequence (the 3D
    record sweep, the plain 3D sweep of odd row lengths and the 2D 32 x 64
    tile sweep; iterates rotating through S + 2 buffers for S iterations in
    flight, 3 in 3D and up to 14 in 2D, speculative iterations past the
    converged one discarded): per-axis periodic / zero-gradient faces,
    several tiles along periodic axes, ragged tiles, iteration caps of 1-7
    and convergence after a few or many host batches.  2D meshes run both
    2D paths: the persistent wavefront of 32-row warps (k_march_gs, walking
    along x, or along y when only y is periodic or both are and y is
    longer; forced with SIFV_GS_MARCH=1) and the tiled sweeps
    (SIFV_GS_MARCH=0).  The iteration count and the whole returned array --
    interior and the ghost layers the reference's last fill leaves -- are
    the oracle's bit for bit."""
    if shape[2] > 1 and not march:
        pytest.skip("3D meshes have one path")
    monkeypatch.setenv("SIFV_GS_MARCH", "1" if march else "0")
    cfg, mesh, fields = cases.acoustic_box(*shape)
    mesh.bc = [bcs[0]] * 2 + [bcs[1]] * 2 + [bcs[2]] * 2
    cg = backends.make(backends.cuda(), (cfg, mesh, fields))
    co = backends.make(backends.oracle(), (cfg, mesh, fields))
    cg.set_pressure_solver(abi.PRESSURE_GAUSS_SEIDEL)
    co.set_pressure_solver(abi.PRESSURE_GAUSS_SEIDEL)
    rng = np.random.default_rng(max_iter + 17 * bcs[0])
    n = cg.ncells
    args = (1.0 + 0.1 * rng.random(n), 1.4 + 0.2 * rng.random(n), rng.random(n), rng.random(n))
    pg, ig, _ = cg.pressure_solve(*args, dt, tol, max_iter)
    po, io, _ = co.pressure_solve(*args, dt, tol, max_iter)
    assert ig == io, (ig, io)
    assert np.array_equal(pg.view(np.int64), po.view(np.int64))


def test_gauss_seidel_standalone_solve():
    case = cases.acoustic3d(12)
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    cg.set_pressure_solver(1)
    co.set_pressure_solver(1)
    rng = np.random.default_rng(12)
    n = cg.ncells
    rho = 1.0 + 0.1 * rng.random(n)
    rhoc2 = 1.4 + 0.2 * rng.random(n)
    rhs = rng.random(n)
    p0 = rng.random(n)
    pg, ig, _ = cg.pressure_solve(rho, rhoc2, rhs, p0, 1e-2, 1e-12, 60)
    po, io, _ = co.pressure_solve(rho, rhoc2, rhs, p0, 1e-2, 1e-12, 60)
    assert ig == io
    assert np.array_equal(cg.interior(pg), co.interior(po))


@pytest.mark.parametrize("name", cases.VISCOUS_CASES)
def test_viscous_stress(name):
    """addViscousFluxes (src/ViscousFlux.cpp:24-303) on every face and the
    viscous step limit (computeViscousDt, src/RKTimeStepping.cpp:161-188),
    explicit and semi-implicit, scalar and per-phase viscosity:
    bit-identical to the oracle."""
    case, n = cases.viscous(name)
    check(case, n)


def test_viscous_3d_explicit_walls():
    """All three face directions with transverse gradients through the
    corner ghosts (no-slip walls on every side), RK2, LF."""
    case = cases.acoustic3d(9, semi=False, igr=False, rk=2, riemann=abi.LF)
    case[0].mu = 0.03
    case[1].bc = [abi.BC_NOSLIPWALL, abi.BC_SLIPWALL, abi.BC_NOSLIPWALL, abi.BC_OUTFLOW,
                  abi.BC_SYMMETRY, abi.BC_NOSLIPWALL]
    check(case, 4)


def test_viscous_advance_matches_step():
    case, _ = cases.viscous("riemann2d_noslip")
    c1 = backends.make(backends.cuda(), case)
    c2 = backends.make(backends.cuda(), case)
    t1, s1, _ = cases.run_steps(c1, 5, t_end=0.05)
    t2, s2 = c2.advance(0, 0.0, 0.05, 5)
    assert s1 == s2 and t1 == t2
    for fid in (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE):
        assert np.array_equal(c1.get_field(fid), c2.get_field(fid))


def test_viscous_rejected_outside_reference_precision():
    case, _ = cases.viscous("vortex_periodic")
    case[0].precision = abi.PREC_FP64_FAST
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(case[0], case[1])
    assert e.value.status == abi.ERR_UNSUPPORTED
    case[0].precision = abi.PREC_FP64
    case[0].mu = -1.0
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(case[0], case[1])
    assert e.value.status == abi.ERR_BAD_CONFIG


@pytest.mark.parametrize("name", cases.CAPILLARY_CASES)
def test_surface_tension(name):
    """addSurfaceTensionFluxes (src/SurfaceTension.cpp:8-254) on every face
    and the capillary step limit (computeCapillaryDt,
    src/RKTimeStepping.cpp:201-228), explicit and semi-implicit, 2D and 3D,
    alone and after the viscous stress: bit-identical to the oracle."""
    case, n = cases.capillary(name)
    check(case, n)


def test_surface_tension_rejected_without_phases():
    case, _ = cases.viscous("vortex_periodic")
    case[0].mu = 0.0
    case[0].stSigma = 0.07
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(case[0], case[1])
    assert e.value.status == abi.ERR_BAD_CONFIG


@pytest.mark.parametrize("name", cases.IB_CASES)
def test_immersed_boundary(name):
    """ImmersedBoundaryMethod on the GPU: cell classification, the ghost-cell
    fill per stage (parallel, or in list order when a stencil reads another
    ghost cell), solid cells out of the update, the dt limit and the IGR
    sweeps; bit-identical to the oracle."""
    case, bodies, n = cases.immersed(name)
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    cg.set_immersed_bodies(bodies)
    co.set_immersed_bodies(bodies)
    assert np.array_equal(cg.ib_cell_types(), co.ib_cell_types())
    check_pair = run_pair_contexts(cg, co, n)
    assert check_pair


def run_pair_contexts(cg, co, n):
    _, _, dtg = cases.run_steps(cg, n)
    _, _, dto = cases.run_steps(co, n)
    assert dtg == dto
    for fid in _fields(cg.cfg):
        assert np.array_equal(cg.get_field(fid), co.get_field(fid)), fid
    return True


def test_immersed_boundary_time_loop_and_removal():
    """The device-resident time loop runs the ghost-cell fill too, and an
    empty body list restores the plain step."""
    case, bodies, _ = cases.immersed("circle_noslip")
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    cg.set_immersed_bodies(bodies)
    co.set_immersed_bodies(bodies)
    st, r = cg.run_time_loop(0.05, 0.02, batch=4)
    t, n = cases.run_time_loop(co, 0.05, 0.02)
    assert st == abi.OK and r.steps == n and r.time == t
    for fid in _fields(case[0]):
        assert np.array_equal(cg.get_field(fid), co.get_field(fid)), fid
    cg.set_immersed_bodies([])
    co.set_immersed_bodies([])
    assert not cg.ib_cell_types().any()
    _, _, dtg = cases.run_steps(cg, 3, step0=n, time0=t)
    _, _, dto = cases.run_steps(co, 3, step0=n, time0=t)
    assert dtg == dto
    for fid in _fields(case[0]):
        assert np.array_equal(cg.get_field(fid), co.get_field(fid)), fid


def test_immersed_boundary_rejected_where_unsupported():
    case, bodies, _ = cases.immersed("circle_noslip")
    semi = cases.acoustic3d(8)
    cs = backends.make(backends.cuda(), semi)
    with pytest.raises(abi.AbiError) as e:
        cs.set_immersed_bodies([abi.ib_body(abi.IB_PRISM, [0.5, 0.5, 0.5, 0.1, 0.1, 0.1])])
    assert e.value.status == abi.ERR_UNSUPPORTED
    case[0].precision = abi.PREC_FP64_FAST
    cf = backends.make(backends.cuda(), case)
    with pytest.raises(abi.AbiError) as e:
        cf.set_immersed_bodies(bodies)
    assert e.value.status == abi.ERR_UNSUPPORTED


@pytest.mark.parametrize("kind", [abi.PRESSURE_JACOBI, abi.PRESSURE_GAUSS_SEIDEL])
def test_standalone_solve_with_more_iterations_than_the_config(kind):
    """A standalone solve allowed more iterations than maxPressureIters grows
    the residual history and keeps dt."""
    case = cases.acoustic3d(10)
    case[0].maxPressureIters = 20
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    cg.set_pressure_solver(kind)
    co.set_pressure_solver(kind)
    rng = np.random.default_rng(5)
    n = cg.ncells
    args = (1.0 + 0.1 * rng.random(n), 1.4 + 0.2 * rng.random(n), rng.random(n), rng.random(n))
    pg, ig, _ = cg.pressure_solve(*args, 0.1, 1e-12, 500)
    po, io, _ = co.pressure_solve(*args, 0.1, 1e-12, 500)
    assert ig == io and ig > 20
    assert np.array_equal(cg.interior(pg), co.interior(po))
