"""Initial conditions of the parity cases, restated from the reference's
example drivers and the configurations the benchmark is quoted on.

Each builder returns ``(cfg, mesh, fields)`` where ``fields`` maps a field
id to a full (ghosts included, ghosts zero) float64 array, so that every
backend receives bit-identical inputs.  Conservative fields are computed the
way the examples compute them (EOS toConservative / mixtureTotalEnergy),
operation for operation, in float64 numpy.
"""
from __future__ import annotations

import numpy as np

from semiimplicitfv_b200 import abi
from semiimplicitfv_b200.abi import (BC_OUTFLOW, BC_PERIODIC, F_ALPHA, F_ALPHARHO, F_PRES, F_RHO, F_RHOE,
                                     F_RHOU, F_RHOV, F_RHOW, F_SIGMA, F_VELU, F_VELV, F_VELW)


def _ext_shape(cfg, nx, ny, nz):
    g = cfg.nGhost
    return (nz + 2 * g if cfg.dim >= 3 else 1, ny + 2 * g if cfg.dim >= 2 else 1, nx + 2 * g)


def _interior_slices(cfg):
    g = cfg.nGhost
    sk = slice(g, -g) if cfg.dim >= 3 else slice(0, 1)
    sj = slice(g, -g) if cfg.dim >= 2 else slice(0, 1)
    return sk, sj, slice(g, -g)


def _centroids(nodes):
    return 0.5 * (nodes[:-1] + nodes[1:])


def _single_phase_fields(cfg, shape, rho, u, v, w, p, eos_gamma, eos_pinf=0.0, stiffened=False):
    """setPrimitiveState + setConservativeState(eos.toConservative(W)) on the
    interior (IdealGasEOS::toConservative src/IdealGasEOS.cpp:66-82,
    StiffenedGasEOS::toConservative src/StiffenedGasEOS.cpp:66-82)."""
    dim = cfg.dim
    sl = _interior_slices(cfg)
    f = {}
    z = lambda: np.zeros(shape)
    for fid in (F_RHO, F_RHOU, F_RHOE, F_VELU, F_PRES, F_SIGMA):
        f[fid] = z()
    if dim >= 2:
        f[F_RHOV], f[F_VELV] = z(), z()
    if dim >= 3:
        f[F_RHOW], f[F_VELW] = z(), z()
    f[F_RHO][sl] = rho
    f[F_VELU][sl] = u
    f[F_PRES][sl] = p
    f[F_RHOU][sl] = rho * u
    ke = 0.0 + u * u
    if dim >= 2:
        f[F_VELV][sl] = v
        f[F_RHOV][sl] = rho * v
        ke = ke + v * v
    if dim >= 3:
        f[F_VELW][sl] = w
        f[F_RHOW][sl] = rho * w
        ke = ke + w * w
    ke = ke * (0.5 * rho)
    if stiffened:
        e = (p + eos_gamma * eos_pinf) / (eos_gamma - 1.0)
    else:
        e = p / (eos_gamma - 1.0)
    f[F_RHOE][sl] = e + ke
    return f


def sod(n=1000, cfl=0.6, recon=abi.WENO5, riemann=abi.HLLC, ng=3, rk=3):
    """1D Sod shock tube (examples/1D_sod_shocktube/1D_sod_shocktube.cpp:24-50):
    x in [0,1], (rho,u,p) = (1,0,1) for x_c < 0.5 else (0.125,0,0.1)."""
    cfg = abi.config_defaults(dim=1, nGhost=ng, RKOrder=rk, reconOrder=recon, riemannSolver=riemann, cfl=cfl)
    x = abi.linspace_nodes(n, 0.0, 1.0)
    xc = _centroids(x)
    left = xc < 0.5
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    u = np.zeros(n)
    shape = _ext_shape(cfg, n, 1, 1)
    fields = _single_phase_fields(cfg, shape, rho[None, None, :], u[None, None, :], None, None,
                                  p[None, None, :], 1.4)
    return cfg, abi.MeshSpec(x, bc=[BC_OUTFLOW] * 6), fields


RIEMANN2D_STATES = {  # (rho, u, v, p) per quadrant, split at (0.8, 0.8)
    "q1": (1.5, 0.0, 0.0, 1.5),
    "q2": (0.5323, 1.206, 0.0, 0.3),
    "q3": (0.138, 1.206, 1.206, 0.029),
    "q4": (0.5323, 0.0, 1.206, 0.3),
}


def riemann2d(n=64, cfl=0.6, recon=abi.WENO5, riemann=abi.HLLC, ng=3, weno_eps=1e-6, bc=BC_OUTFLOW, rk=3):
    """2D four-quadrant Riemann problem (examples/2D_riemann/2D_riemann.cpp:24-76
    with the 0.5323 states of the benchmark configuration)."""
    cfg = abi.config_defaults(dim=2, nGhost=ng, RKOrder=rk, reconOrder=recon, riemannSolver=riemann, cfl=cfl,
                              wenoEps=weno_eps)
    x = abi.linspace_nodes(n, 0.0, 1.0)
    y = abi.linspace_nodes(n, 0.0, 1.0)
    X, Y = np.meshgrid(_centroids(x), _centroids(y), indexing="xy")
    q = np.empty(X.shape, dtype=object)
    rho = np.empty(X.shape); u = np.empty(X.shape); v = np.empty(X.shape); p = np.empty(X.shape)
    for name, mask in (("q1", (X >= 0.8) & (Y >= 0.8)), ("q2", (X < 0.8) & (Y >= 0.8)),
                       ("q3", (X < 0.8) & (Y < 0.8)), ("q4", (X >= 0.8) & (Y < 0.8))):
        r_, u_, v_, p_ = RIEMANN2D_STATES[name]
        rho[mask], u[mask], v[mask], p[mask] = r_, u_, v_, p_
    shape = _ext_shape(cfg, n, n, 1)
    fields = _single_phase_fields(cfg, shape, rho[None], u[None], v[None], None, p[None], 1.4)
    return cfg, abi.MeshSpec(x, y, bc=[bc] * 6), fields


def acoustic3d(n=16, semi=True, igr=True, rk=1, recon=abi.WENO5, riemann=abi.HLLC, ng=3, tol=1e-6,
               max_iter=1000, alpha_coeff=10.0, igr_iters=5, warm=50):
    """3D low-Mach acoustic pulse on the periodic unit cube:
    rho = 1, u = (0.1, 0.05, 0), p = 1 + 1e-3 exp(-|x - 0.5|^2 / 0.01)."""
    cfg = abi.config_defaults(dim=3, nGhost=ng, RKOrder=rk, reconOrder=recon, riemannSolver=riemann,
                              semiImplicit=int(semi), useIGR=int(igr), siCfl=0.8, pressureTol=tol,
                              maxPressureIters=max_iter, alphaCoeff=alpha_coeff, IGRIters=igr_iters,
                              IGRWarmStartIters=warm)
    x = abi.linspace_nodes(n, 0.0, 1.0)
    c = _centroids(x)
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    r2 = (X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2
    p = 1.0 + 1e-3 * np.exp(-r2 / 0.01)
    rho = np.ones_like(p)
    u = np.full_like(p, 0.1); v = np.full_like(p, 0.05); w = np.zeros_like(p)
    shape = _ext_shape(cfg, n, n, n)
    fields = _single_phase_fields(cfg, shape, rho, u, v, w, p, 1.4)
    return cfg, abi.MeshSpec(x, x, x, bc=[BC_PERIODIC] * 6), fields


def acoustic_box(nx, ny, nz=1, semi=True, igr=True, rk=1, bc=BC_PERIODIC, stretch=0.0, max_iter=300, tol=1e-8):
    """Low-Mach acoustic pulse on a box of nx x ny (x nz) cells, [0,1] per
    axis, optionally with geometrically stretched x nodes (ratio 1 + stretch
    per cell); dim = 3 when nz > 1 else 2.  Same state as acoustic3d."""
    dim = 3 if nz > 1 else 2
    cfg = abi.config_defaults(dim=dim, nGhost=3, RKOrder=rk, reconOrder=abi.WENO5, riemannSolver=abi.HLLC,
                              semiImplicit=int(semi), useIGR=int(igr), siCfl=0.8, pressureTol=tol,
                              maxPressureIters=max_iter, alphaCoeff=10.0, IGRIters=5, IGRWarmStartIters=20)
    if stretch > 0:
        w = (1.0 + stretch) ** np.arange(nx)
        x = np.concatenate([[0.0], np.cumsum(w) / np.sum(w)])
    else:
        x = abi.linspace_nodes(nx, 0.0, 1.0)
    y = abi.linspace_nodes(ny, 0.0, 1.0)
    z = abi.linspace_nodes(nz, 0.0, 1.0) if dim == 3 else None
    cx, cy = _centroids(x), _centroids(y)
    if dim == 3:
        Z, Y, X = np.meshgrid(_centroids(z), cy, cx, indexing="ij")
        r2 = (X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2
    else:
        Y, X = np.meshgrid(cy, cx, indexing="ij")
        r2 = ((X - 0.5) ** 2 + (Y - 0.5) ** 2)[None]
    p = 1.0 + 1e-3 * np.exp(-r2 / 0.01)
    rho = np.ones_like(p)
    u = np.full_like(p, 0.1)
    v = np.full_like(p, 0.05)
    w = np.zeros_like(p)
    shape = _ext_shape(cfg, nx, ny, nz)
    fields = _single_phase_fields(cfg, shape, rho, u, v, w if dim == 3 else None, p, 1.4)
    mesh = abi.MeshSpec(x, y, z, bc=[bc] * 6) if dim == 3 else abi.MeshSpec(x, y, bc=[bc] * 6)
    return cfg, mesh, fields


def vortex2d(n=512, beta=5.0, L=10.0, cfl=0.6, recon=abi.WENO5, riemann=abi.HLLC, rk=3):
    """Isentropic vortex (Shu; examples/2D_isentropic_vortex/2D_isentropic_vortex.cpp:65-94)
    on the periodic square [-L/2, L/2]^2 centred at the origin, free stream
    (rho, u, v, p) = (1, 1, 1, 1), R = 1 (T_inf = 1), gamma 1.4."""
    g = 1.4
    cfg = abi.config_defaults(dim=2, nGhost=3, RKOrder=rk, reconOrder=recon, riemannSolver=riemann, cfl=cfl,
                              maxDt=1.0)
    x = abi.linspace_nodes(n, -0.5 * L, 0.5 * L)
    c = _centroids(x)
    X, Y = np.meshgrid(c, c, indexing="xy")
    dx = X - L * np.round(X / L)
    dy = Y - L * np.round(Y / L)
    r2 = dx * dx + dy * dy
    f = np.exp(0.5 * (1.0 - r2))
    f2 = np.exp(1.0 - r2)
    du = -beta / (2.0 * np.pi) * dy * f
    dv = beta / (2.0 * np.pi) * dx * f
    dT = -(g - 1.0) * beta * beta / (8.0 * g * np.pi * np.pi) * f2
    T = 1.0 + dT
    rho = T ** (1.0 / (g - 1.0))
    p = T ** (g / (g - 1.0))
    shape = _ext_shape(cfg, n, n, 1)
    fields = _single_phase_fields(cfg, shape, rho[None], (1.0 + du)[None], (1.0 + dv)[None], None, p[None], g)
    return cfg, abi.MeshSpec(x, x, bc=[BC_PERIODIC] * 6), fields


def water_air(n=256, x_interface=0.5, p_left=5e8, rho_air=1.0, cfl=0.5, recon=abi.WENO5, riemann=abi.HLLC,
              ng=3, alpha_min=1e-8, rk=3):
    """1D two-phase water-air shock tube (examples/1D_liquid_gas_shocktube/
    1D_liquid_gas_shocktube.cpp:34-77): water gamma 4.4, pInf 6e8, rho 1000 at
    p_left left of the interface; air gamma 1.4, rho_air, p 1e5 right."""
    cfg = abi.config_defaults(dim=1, nGhost=ng, RKOrder=rk, reconOrder=recon, riemannSolver=riemann, cfl=cfl,
                              nPhases=2, phaseGamma=[4.4, 1.4], phasePInf=[6.0e8, 0.0], alphaMin=alpha_min)
    x = abi.linspace_nodes(n, 0.0, 1.0)
    xc = _centroids(x)
    left = xc < x_interface
    rho = np.where(left, 1000.0, rho_air)
    p = np.where(left, p_left, 1.0e5)
    aw = np.where(left, 1.0 - alpha_min, alpha_min)
    aa = 1.0 - aw
    shape = _ext_shape(cfg, n, 1, 1)
    sl = _interior_slices(cfg)
    f = {fid: np.zeros(shape) for fid in (F_RHO, F_RHOU, F_RHOE, F_VELU, F_PRES, F_SIGMA,
                                          F_ALPHARHO(0), F_ALPHARHO(1), F_ALPHA(0), F_ALPHA(1))}
    ar0, ar1 = aw * rho, aa * rho
    f[F_ALPHARHO(0)][sl] = ar0
    f[F_ALPHARHO(1)][sl] = ar1
    f[F_ALPHA(0)][sl] = aw
    f[F_ALPHA(1)][sl] = aa
    f[F_RHO][sl] = ar0 + ar1
    f[F_PRES][sl] = p
    # mixtureTotalEnergy(rho, p, alphas, ke=0) (src/MixtureEOS.cpp:65-76)
    e = 0.0 + aw * (p + 4.4 * 6.0e8) / (4.4 - 1.0)
    e = e + aa * (p + 1.4 * 0.0) / (1.4 - 1.0)
    f[F_RHOE][sl] = e
    return cfg, abi.MeshSpec(x, bc=[BC_OUTFLOW] * 6), f


def advection1d(n=128, semi=False, riemann=abi.LF, cfl=0.8, rk=3):
    """1D periodic density-pulse advection (examples/1D_advection/1D_advection.cpp:36-67,
    85-99): rho0 = 1.225 (1 + 0.01 exp(-d^2 / 0.05^2)), u = 10, p = 101325."""
    rho0, p0, u0, amp, xcen, sig = 1.225, 101325.0, 10.0, 0.01, 0.5, 0.05
    if semi:
        cfg = abi.config_defaults(dim=1, nGhost=3, RKOrder=rk, reconOrder=abi.WENO5, riemannSolver=riemann,
                                  semiImplicit=1, siCfl=cfl, siMaxDt=1e-2, pressureTol=1e-9, maxPressureIters=200,
                                  alphaCoeff=10.0, IGRIters=5)
    else:
        cfg = abi.config_defaults(dim=1, nGhost=3, RKOrder=rk, reconOrder=abi.WENO5, riemannSolver=riemann, cfl=cfl,
                                  maxDt=1e-2)
    x = abi.linspace_nodes(n, 0.0, 1.0)
    xc = _centroids(x)
    d = xc - xcen
    d = d - 1.0 * np.round(d / 1.0)
    rho = rho0 * (1.0 + amp * np.exp(-(d * d) / (sig * sig)))
    shape = _ext_shape(cfg, n, 1, 1)
    fields = _single_phase_fields(cfg, shape, rho[None, None, :], np.full((1, 1, n), u0), None, None,
                                  np.full((1, 1, n), p0), 1.4)
    return cfg, abi.MeshSpec(x, bc=[BC_PERIODIC] * 6), fields


def droplet(n=48, dim=2, semi=False, sigma=0.0728, rk=3, bc=BC_OUTFLOW):
    """Water droplet in air with surface tension (examples/2D_laplace_pressure_jump/
    2D_laplace_pressure_jump.cpp:39-83): radius 1 mm in [0, 6 mm]^dim, water
    gamma 4.4 / pInf 6e8 / rho 1000, air gamma 1.4 / rho 1.225, interface
    alpha_w = (1 - tanh((r - R0) / 3 dx)) / 2 clipped to [alphaMin, 1 - alphaMin],
    energy from p = pAtm + (sigma / R0) alpha-profile, stored pressure pAtm,
    fluid at rest.  dim = 3 puts a sphere in the cube."""
    L, R0, p_atm, rw, ra, amin = 6.0e-3, 1.0e-3, 1.0e5, 1000.0, 1.225, 1e-8
    cfg = abi.config_defaults(dim=dim, nGhost=3, RKOrder=rk, reconOrder=abi.WENO5, riemannSolver=abi.HLLC,
                              cfl=0.5, semiImplicit=int(semi), siCfl=0.5, pressureTol=1e-3, maxPressureIters=200,
                              nPhases=2, phaseGamma=[4.4, 1.4], phasePInf=[6.0e8, 0.0], alphaMin=amin,
                              stSigma=sigma)
    x = abi.linspace_nodes(n, 0.0, L)
    c = _centroids(x)
    if dim == 3:
        Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
        r = np.sqrt((X - 0.5 * L) ** 2 + (Y - 0.5 * L) ** 2 + (Z - 0.5 * L) ** 2)
    else:
        Y, X = np.meshgrid(c, c, indexing="ij")
        r = np.sqrt((X - 0.5 * L) ** 2 + (Y - 0.5 * L) ** 2)[None]
    eps = 3.0 * (x[1] - x[0])
    prof = 0.5 * (1.0 - np.tanh((r - R0) / eps))
    aw = np.maximum(amin, np.minimum(1.0 - amin, prof))
    aa = 1.0 - aw
    p = p_atm + (0.0728 / R0) * prof   # Laplace jump sigma / R0 of water-air
    shape = _ext_shape(cfg, n, n if dim >= 2 else 1, n if dim >= 3 else 1)
    sl = _interior_slices(cfg)
    fids = [F_RHO, F_RHOU, F_RHOV, F_RHOE, F_VELU, F_VELV, F_PRES, F_SIGMA,
            F_ALPHARHO(0), F_ALPHARHO(1), F_ALPHA(0), F_ALPHA(1)]
    if dim >= 3:
        fids += [F_RHOW, F_VELW]
    f = {fid: np.zeros(shape) for fid in fids}
    f[F_ALPHARHO(0)][sl] = aw * rw
    f[F_ALPHARHO(1)][sl] = aa * ra
    f[F_ALPHA(0)][sl] = aw
    f[F_ALPHA(1)][sl] = aa
    f[F_RHO][sl] = aw * rw + aa * ra
    f[F_PRES][sl] = p_atm
    # mixtureTotalEnergy(rho, p, alphas, ke=0) (src/MixtureEOS.cpp:65-76)
    e = 0.0 + aw * (p + 4.4 * 6.0e8) / (4.4 - 1.0)
    e = e + aa * (p + 1.4 * 0.0) / (1.4 - 1.0)
    f[F_RHOE][sl] = e
    mesh = abi.MeshSpec(x, x, x, bc=[bc] * 6) if dim == 3 else abi.MeshSpec(x, x, bc=[bc] * 6)
    return cfg, mesh, f


CAPILLARY_CASES = ["droplet2d", "droplet2d_semi", "droplet3d_walls", "droplet2d_viscous"]


def capillary(name):
    """Surface-tension variants (surfaceTensionParams, include/SimulationConfig.hpp:67-70).
    Returns (case, steps)."""
    if name == "droplet2d":
        return droplet(40), 5
    if name == "droplet2d_semi":
        return droplet(32, semi=True, rk=2), 3
    if name == "droplet3d_walls":
        c = droplet(14, dim=3, rk=2)
        c[1].bc = [abi.BC_NOSLIPWALL, abi.BC_SLIPWALL, abi.BC_OUTFLOW, abi.BC_SYMMETRY,
                   abi.BC_NOSLIPWALL, abi.BC_OUTFLOW]
        return c, 3
    if name == "droplet2d_viscous":
        c = droplet(32, bc=abi.BC_PERIODIC)
        c[0].nPhaseMu = 2
        c[0].phaseMu[0], c[0].phaseMu[1] = 1.0e-3, 1.8e-5
        c[0].mu = 1.0e-4
        c[0].stEpsGradAlpha = 1e-3
        return c, 4
    raise KeyError(name)


def flow_over_circle(nx=40, ny=20, slip=False, igr=False):
    """Uniform Mach 0.2 stream past a circle (examples/2D_flow_over_circle/
    2D_flow_over_circle.cpp:19-170): [0, 4] x [0, 2], circle (1, 1) r 0.2,
    rho 1, u 1, p = 1 / (1.4 M^2); x outflow, y slip walls; cfl 0.5,
    maxDt 1; IGR alphaCoeff 1.  Returns (case, bodies)."""
    cfg = abi.config_defaults(dim=2, nGhost=3, RKOrder=3, reconOrder=abi.WENO5, riemannSolver=abi.HLLC,
                              cfl=0.5, maxDt=1.0, useIGR=int(igr), alphaCoeff=1.0, IGRIters=5,
                              IGRWarmStartIters=50)
    x = abi.linspace_nodes(nx, 0.0, 4.0)
    y = abi.linspace_nodes(ny, 0.0, 2.0)
    p_inf = 1.0 / (1.4 * 0.2 * 0.2)
    shape = _ext_shape(cfg, nx, ny, 1)
    one = np.ones((1, ny, nx))
    fields = _single_phase_fields(cfg, shape, one, one, 0.0 * one, None, p_inf * one, 1.4)
    mesh = abi.MeshSpec(x, y, bc=[BC_OUTFLOW, BC_OUTFLOW, abi.BC_SLIPWALL, abi.BC_SLIPWALL, 0, 0])
    body = abi.ib_body(abi.IB_CIRCLE, [1.0, 1.0, 0.2], abi.IB_SLIP if slip else abi.IB_NOSLIP)
    return (cfg, mesh, fields), [body]


IB_CASES = ["circle_noslip", "circle_slip_igr", "rectangle_riemann", "prism_cylinder_3d", "droplet_rectangle",
            "two_circles_1d", "slit_sequential"]


def immersed(name):
    """Immersed-boundary cases: (case, bodies, steps)."""
    if name == "circle_noslip":
        case, bodies = flow_over_circle(48, 24)
        return case, bodies, 6
    if name == "circle_slip_igr":
        case, bodies = flow_over_circle(40, 20, slip=True, igr=True)
        return case, bodies, 3
    if name == "rectangle_riemann":
        case = riemann2d(36, bc=abi.BC_SLIPWALL)
        return case, [abi.ib_body(abi.IB_RECTANGLE, [0.45, 0.55, 0.12, 0.08], abi.IB_SLIP),
                      abi.ib_body(abi.IB_CIRCLE, [0.7, 0.3, 0.09])], 6
    if name == "prism_cylinder_3d":
        case = acoustic3d(14, semi=False, igr=False, rk=2)
        case[1].bc = [abi.BC_OUTFLOW, abi.BC_SLIPWALL, abi.BC_NOSLIPWALL, abi.BC_OUTFLOW,
                      abi.BC_SYMMETRY, abi.BC_OUTFLOW]
        return case, [abi.ib_body(abi.IB_PRISM, [0.3, 0.35, 0.5, 0.12, 0.1, 0.2], abi.IB_SLIP),
                      abi.ib_body(abi.IB_CYLINDER, [0.7, 0.6, 0.13], abi.IB_NOSLIP, axis=1)], 4
    if name == "droplet_rectangle":
        case = droplet(24)
        return case, [abi.ib_body(abi.IB_RECTANGLE, [1.2e-3, 3.0e-3, 4e-4, 1.5e-3], abi.IB_NOSLIP)], 4
    if name == "two_circles_1d":
        case = water_air(64, p_left=2e5)
        return case, [abi.ib_body(abi.IB_CIRCLE, [0.25, 0.5, 0.06]),
                      abi.ib_body(abi.IB_CIRCLE, [0.8, 0.5, 0.05], abi.IB_SLIP)], 6
    if name == "slit_sequential":   # a sub-cell slit: some stencils see only ghost cells
        case = riemann2d(40, bc=abi.BC_SLIPWALL)
        return case, [abi.ib_body(abi.IB_RECTANGLE, [0.3, 0.5, 0.1, 0.2]),
                      abi.ib_body(abi.IB_RECTANGLE, [0.51, 0.5, 0.1, 0.2], abi.IB_SLIP)], 5
    raise KeyError(name)


VISCOUS_CASES = ["riemann2d_noslip", "water_air_phase_mu", "acoustic3d_semi", "vortex_periodic"]


def viscous(name):
    """Viscous variants (viscousParams, include/SimulationConfig.hpp:62-65):
    scalar mu on the no-slip 2D Riemann box, per-phase mu on water-air,
    scalar mu on the semi-implicit 3D pulse and on the periodic vortex.
    Returns (case, steps)."""
    if name == "riemann2d_noslip":
        c = riemann2d(32, bc=abi.BC_NOSLIPWALL)
        c[0].mu = 0.01
        return c, 6
    if name == "water_air_phase_mu":
        c = water_air(64, p_left=2e5)
        c[0].nPhaseMu = 2
        c[0].phaseMu[0], c[0].phaseMu[1] = 1.0e-3, 1.8e-5
        return c, 6
    if name == "acoustic3d_semi":
        c = acoustic3d(10, igr=False)
        c[0].mu = 0.05
        return c, 3
    if name == "vortex_periodic":
        c = vortex2d(32)
        c[0].mu = 0.02
        return c, 4
    raise KeyError(name)


def run_steps(ctx, nsteps, t_end=None, step0=0, time0=0.0):
    """Drive ctx.step like the reference drivers: targetDt = t_end - t when
    given.  Returns (time, steps, dts)."""
    t, s, dts = time0, step0, []
    while s - step0 < nsteps and (t_end is None or t < t_end):
        target = (t_end - t) if t_end is not None else -1.0
        dt = ctx.step(s, t, target)
        dts.append(dt)
        t += dt
        s += 1
    return t, s, dts


def run_time_loop(ctx, t_end, output_interval, on_output=None, print_interval=None, on_print=None):
    """runTimeLoop (src/RKTimeStepping.cpp:241-356): output at t = 0 and when
    t >= nextOutput - 1e-12 outputInterval, targetDt clamped to the next
    output time, config.step incremented per step; on_output(time, step)
    at each output, on_print(step, time, dt) at step 1 and every
    print_interval-th step."""
    if on_output:
        on_output(0.0, 0)
    time, step = 0.0, 0
    next_out = output_interval
    while time < t_end:
        target = t_end - time
        if next_out < t_end:
            target = min(target, next_out - time)
        dt = ctx.step(step, time, target)
        time += dt
        step += 1
        if time >= next_out - 1e-12 * output_interval:
            if on_output:
                on_output(time, step)
            next_out += output_interval
        if on_print and (step % print_interval == 0 or step == 1):
            on_print(step, time, dt)
    return time, step


def output_fields(ctx, cfg):
    """The fields a VTK snapshot of ``ctx`` reads, as SIFV_F_* -> array."""
    ids = [abi.F_PRES, abi.F_RHOE, abi.F_VELU, abi.F_RHOU]
    if cfg.useIGR:
        ids.append(abi.F_SIGMA)
    if cfg.dim >= 2:
        ids += [abi.F_VELV, abi.F_RHOV]
    if cfg.dim >= 3:
        ids += [abi.F_VELW, abi.F_RHOW]
    if cfg.nPhases == 0:
        ids.append(abi.F_RHO)
    for p in range(cfg.nPhases):
        ids += [abi.F_ALPHARHO(p), abi.F_ALPHA(p)]
    return {fid: ctx.get_field(fid) for fid in ids}
