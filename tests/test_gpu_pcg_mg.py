"""The PCG + multigrid pressure solver (SIFV_PRESSURE_PCG_MG), the CUDA
counterpart of the reference's Hypre PCG+PFMG solver: it must solve the
system HyprePressureSolver assembles (oracle/hypre_system.py, checked by a
sparse direct solve) to the reference's stopping rule |A p - b| <= tol |b|,
with iteration counts that stay nearly flat as the mesh is refined, and a
semi-implicit step that uses it must agree with one converged by the
reference-ordered Gauss-Seidel solver."""
import os
import sys

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import hypre_system  # noqa: E402

pytestmark = pytest.mark.gpu


def _system_case(name):
    """(cfg, mesh, periodic flags) of the solver test meshes."""
    if name == "1d_outflow":
        cfg = abi.config_defaults(dim=1, nGhost=3, reconOrder=abi.WENO5, semiImplicit=1)
        return cfg, abi.MeshSpec(abi.linspace_nodes(300, 0.0, 1.0)), (False, False, False)
    if name == "2d_periodic":
        cfg = abi.config_defaults(dim=2, nGhost=3, reconOrder=abi.WENO5, semiImplicit=1)
        return cfg, abi.MeshSpec(abi.linspace_nodes(96, 0.0, 1.5), abi.linspace_nodes(64, 0.0, 1.0),
                                 bc=[abi.BC_PERIODIC] * 4 + [0, 0]), (True, True, False)
    if name == "2d_stretched_walls":
        cfg = abi.config_defaults(dim=2, nGhost=3, reconOrder=abi.WENO5, semiImplicit=1)
        w = 1.03 ** np.arange(80)
        x = np.concatenate([[0.0], np.cumsum(w) / w.sum()])
        return cfg, abi.MeshSpec(x, abi.linspace_nodes(72, 0.0, 1.0), bc=[abi.BC_SLIPWALL] * 4 + [0, 0]), \
            (False, False, False)
    if name == "3d_mixed":
        cfg = abi.config_defaults(dim=3, nGhost=3, reconOrder=abi.WENO5, semiImplicit=1)
        bc = [abi.BC_PERIODIC, abi.BC_PERIODIC, abi.BC_OUTFLOW, abi.BC_OUTFLOW, abi.BC_NOSLIPWALL, abi.BC_SLIPWALL]
        return cfg, abi.MeshSpec(abi.linspace_nodes(24, 0.0, 1.0), abi.linspace_nodes(20, 0.0, 1.0),
                                 abi.linspace_nodes(18, 0.0, 0.9), bc=bc), (True, False, False)
    raise KeyError(name)


def _inputs(ctx, periodic, seed):
    rng = np.random.default_rng(seed)
    shape = ctx.shape
    g = ctx.ng
    dim = ctx.cfg.dim
    pads = [(g, g) if dim >= 3 else (0, 0), (g, g) if dim >= 2 else (0, 0), (g, g)]
    inner = tuple(s - a - b for s, (a, b) in zip(shape, pads))

    def field(lo, hi):
        a = lo + (hi - lo) * rng.random(inner)
        out = a
        for ax, (pw, per) in enumerate(zip(pads, (periodic[2], periodic[1], periodic[0]))):
            if pw[0]:
                out = np.pad(out, [(0, 0)] * ax + [pw] + [(0, 0)] * (2 - ax), mode="wrap" if per else "edge")
        return out

    return field(0.5, 2.0), field(1.0, 3.0), rng.standard_normal(shape), rng.standard_normal(shape)


@pytest.mark.parametrize("name", ["1d_outflow", "2d_periodic", "2d_stretched_walls", "3d_mixed"])
def test_pcg_mg_solves_the_hypre_system(name):
    cfg, mesh, periodic = _system_case(name)
    ctx = backends.cuda().create(cfg, mesh)
    ctx.set_pressure_solver(abi.PRESSURE_PCG_MG)
    rho, rhoc2, rhs, p0 = _inputs(ctx, periodic, 7)
    dx = 1.0 / max(ctx.shape)
    dt = 8.0 * dx   # acoustic CFL ~ 10: a stiff system
    tol = 1e-8
    p, iters, st = ctx.pressure_solve(rho, rhoc2, rhs, p0, dt, tol, 200)
    assert st == abi.OK and 0 < iters <= (60 if "stretched" in name else 30), iters
    dim = cfg.dim
    n = (ctx.shape[2] - 2 * ctx.ng, ctx.shape[1] - (2 * ctx.ng if dim >= 2 else 0),
         ctx.shape[0] - (2 * ctx.ng if dim >= 3 else 0))
    ng = (ctx.ng, ctx.ng if dim >= 2 else 0, ctx.ng if dim >= 3 else 0)
    nodes = [mesh.x, mesh.y if mesh.y is not None else np.array([0.0, 1.0]),
             mesh.z if mesh.z is not None else np.array([0.0, 1.0])]
    widths = [hypre_system.ext_widths(nodes[a], ng[a]) for a in range(3)]
    A, b = hypre_system.assemble(dim, n, ng, widths, periodic, rho.ravel(), rhoc2.ravel(), rhs.ravel(), dt)
    x = ctx.interior(p).ravel()
    assert np.linalg.norm(A @ x - b) <= 2.0 * tol * np.linalg.norm(b)
    xs = hypre_system.solve(A, b)
    assert np.linalg.norm(x - xs) <= 1e-5 * np.linalg.norm(xs)
    # ghosts are not written, as the reference copies back interior cells only
    mask = np.ones(ctx.shape, bool)
    mask[ctx.interior_slices()] = False
    assert np.array_equal(p[mask], p0[mask])


def test_pcg_mg_iterations_stay_flat():
    its = []
    for n in (64, 256):
        cfg = abi.config_defaults(dim=2, nGhost=3, reconOrder=abi.WENO5, semiImplicit=1)
        mesh = abi.MeshSpec(abi.linspace_nodes(n, 0.0, 1.0), abi.linspace_nodes(n, 0.0, 1.0),
                            bc=[abi.BC_PERIODIC] * 4 + [0, 0])
        ctx = backends.cuda().create(cfg, mesh)
        ctx.set_pressure_solver(abi.PRESSURE_PCG_MG)
        rho, rhoc2, rhs, p0 = _inputs(ctx, (True, True, False), 3)
        _, iters, st = ctx.pressure_solve(rho, rhoc2, rhs, 0 * p0, 10.0 / n, 1e-8, 500)
        assert st == abi.OK
        its.append(iters)
    assert its[1] <= 2 * its[0] + 2, its


def test_semi_implicit_step_with_pcg_mg_matches_converged_gauss_seidel():
    case = cases.acoustic3d(12)
    case[0].pressureTol = 1e-12
    case[0].maxPressureIters = 20000
    cg = backends.make(backends.cuda(), case)
    co = backends.make(backends.oracle(), case)
    cg.set_pressure_solver(abi.PRESSURE_PCG_MG)
    co.set_pressure_solver(abi.PRESSURE_GAUSS_SEIDEL)
    _, _, dtg = cases.run_steps(cg, 3)
    _, _, dto = cases.run_steps(co, 3)
    assert dtg == dto
    for fid in (abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_PRES, abi.F_SIGMA):
        a, b = cg.interior(cg.get_field(fid)), co.interior(co.get_field(fid))
        scale = np.abs(b).max()
        assert np.abs(a - b).max() <= 1e-8 * scale, fid


def test_standalone_matches_step_and_rejects_unknown_kind():
    case = cases.acoustic3d(8)
    cg = backends.make(backends.cuda(), case)
    with pytest.raises(abi.AbiError) as e:
        cg.set_pressure_solver(7)
    assert e.value.status == abi.ERR_BAD_ARG
    cg.set_pressure_solver(abi.PRESSURE_PCG_MG)
    dt = cg.step(0, 0.0, -1.0)
    assert dt > 0 and cg.last_pressure_iterations() > 0
