"""Discrete adjoint and tangent of the explicit step (sifv_adjoint_*,
sifv_tangent_*).

- Dot-product test: for random seeds lam and directions v,
  <lam, T v> (tangent) equals <T^T lam, v> (adjoint) to round-off, over
  Riemann solvers, reconstructions, RK orders, boundary conditions and
  dimensions (the same linearisation, transposed).
- Finite differences: the gradient of J = sum_{r<1} p^2 dA of the isentropic
  vortex agrees with central differences (h = 1e-6, FP64, the recorded dt
  sequence) to 1e-6 relative on seeded unit directions, through the
  test-side torch.autograd.Function.
"""
import numpy as np
import pytest
import torch

import backends
import cases
from adjoint_autograd import SifvEvolve, cons_fids, pressure
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu


def _interior_mask(ctx):
    m = np.zeros(ctx.shape, dtype=bool)
    ctx.interior(m)[...] = True
    return m


def _dot_test(case, t_end, every=3, seed=0):
    cfg = case[0]
    rng = np.random.default_rng(seed)
    ctx = backends.make(backends.cuda(), case)
    fids = cons_fids(cfg.dim)
    U0 = {f: ctx.get_field(f).copy() for f in fids}
    mask = _interior_mask(ctx)
    lam = {f: np.where(mask, rng.standard_normal(ctx.shape), 0.0) for f in fids}
    v = {f: np.where(mask, rng.standard_normal(ctx.shape), 0.0) for f in fids}
    t, n = ctx.adjoint_forward(0, 0.0, t_end, 0, every)
    assert n >= 2
    sched = ctx.adjoint_schedule()
    for f in fids:
        ctx.adjoint_set_seed(f, lam[f])
    ctx.adjoint_backward()
    g = {f: ctx.adjoint_get_gradient(f) for f in fids}
    # tangent from the same initial state and dt sequence
    for f in fids:
        ctx.set_field(f, U0[f])
        ctx.tangent_set_direction(f, v[f])
    t2, n2 = ctx.tangent_forward(0, 0.0, t_end, 0, sched)
    assert n2 == n
    tv = {f: ctx.tangent_get(f) for f in fids}
    lhs = sum(float(np.sum(lam[f] * tv[f])) for f in fids)
    rhs = sum(float(np.sum(g[f] * v[f])) for f in fids)
    scale = sum(float(np.sum(np.abs(lam[f] * tv[f]))) for f in fids)
    assert np.isfinite(lhs) and np.isfinite(rhs)
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)
    for f in fids:   # ghost entries of the gradient are zero
        assert np.all(g[f][~mask] == 0.0)
    return ctx


@pytest.mark.parametrize("riemann", [abi.HLLC, abi.RUSANOV, abi.LF])
@pytest.mark.parametrize("recon,rk", [(abi.WENO5, 3), (abi.WENO5, 1), (abi.UPWIND5, 2)])
def test_dot_product_1d_sod(riemann, recon, rk):
    _dot_test(cases.sod(64, riemann=riemann, recon=recon, rk=rk), 0.05)


@pytest.mark.parametrize("bc", [abi.BC_PERIODIC, abi.BC_SLIPWALL, abi.BC_SYMMETRY, abi.BC_NOSLIPWALL])
def test_dot_product_2d_boundaries(bc):
    _dot_test(cases.riemann2d(24, bc=bc), 0.05)


def test_dot_product_2d_vortex_periodic():
    _dot_test(cases.vortex2d(32), 0.6)


def test_dot_product_3d():
    _dot_test(cases.acoustic3d(10, semi=False, igr=False, rk=3), 0.02)


def test_state_after_backward_is_forward_end_state():
    case = cases.riemann2d(24)
    c1 = backends.make(backends.cuda(), case)
    c2 = backends.make(backends.cuda(), case)
    c1.adjoint_forward(0, 0.0, 0.05, 0, 2)
    t, n = c2.adjoint_forward(0, 0.0, 0.05, 0, 2)
    for f in cons_fids(2):
        c2.adjoint_set_seed(f, np.ones(c2.shape))
    c2.adjoint_backward()
    for f in cons_fids(2) + [abi.F_VELU, abi.F_VELV, abi.F_PRES]:
        assert np.array_equal(c1.get_field(f), c2.get_field(f))


def test_forward_matches_step():
    """The recorded forward is the plain reference-ordered step sequence."""
    case = cases.riemann2d(32)
    c1 = backends.make(backends.cuda(), case)
    c2 = backends.make(backends.cuda(), case)
    t, n = c1.adjoint_forward(0, 0.0, 0.05, 0, 4)
    t2, n2, dts = cases.run_steps(c2, 10 ** 6, t_end=0.05)
    assert (t, n) == (t2, n2)
    assert np.array_equal(c1.adjoint_schedule(), np.array(dts))
    for f in cons_fids(2):
        assert np.array_equal(c1.get_field(f), c2.get_field(f))


def test_vortex_gradient_matches_central_differences():
    n, t_end = 32, 1.0
    case = cases.vortex2d(n)
    ctx = backends.make(backends.cuda(), case)
    fids = cons_fids(2)
    U0 = torch.stack([torch.from_numpy(ctx.get_field(f).copy()) for f in fids])
    mask = torch.from_numpy(_interior_mask(ctx))
    x = case[1].x
    c = 0.5 * (x[:-1] + x[1:])
    X, Y = np.meshgrid(c, c, indexing="xy")
    disk = np.zeros(ctx.shape)
    ctx.interior(disk)[...] = ((X * X + Y * Y) < 1.0)[None] * (x[1] - x[0]) ** 2
    w = torch.from_numpy(disk)

    def J(U):
        return torch.sum(w * pressure(U) ** 2)

    U = U0.clone().requires_grad_(True)
    UN = SifvEvolve.apply(U, ctx, t_end, None, 4)
    sched = ctx.adjoint_schedule()
    assert len(sched) >= 8
    J(UN).backward()
    grad = U.grad
    rng = np.random.default_rng(20261203)
    h = 1e-6
    worst = 0.0
    for _ in range(6):
        v = torch.from_numpy(rng.standard_normal(U0.shape)) * mask
        v = v / torch.linalg.norm(v)
        with torch.no_grad():
            jp = J(SifvEvolve.apply(U0 + h * v, ctx, t_end, sched, 1000))
            jm = J(SifvEvolve.apply(U0 - h * v, ctx, t_end, sched, 1000))
        fd = float((jp - jm) / (2 * h))
        ad = float(torch.sum(grad * v))
        rel = abs(fd - ad) / max(abs(fd), abs(ad))
        worst = max(worst, rel)
    assert worst <= 1e-6, worst


def test_adjoint_rejects_unsupported():
    case = cases.water_air(32)
    ctx = backends.make(backends.cuda(), case)
    with pytest.raises(abi.AbiError) as e:
        ctx.adjoint_forward(0, 0.0, 1e-5, 0, 4)
    assert e.value.status == abi.ERR_UNSUPPORTED
    cv, _ = cases.viscous("vortex_periodic")
    ctxv = backends.make(backends.cuda(), cv)
    with pytest.raises(abi.AbiError) as e:
        ctxv.adjoint_forward(0, 0.0, 1e-3, 0, 4)
    assert e.value.status == abi.ERR_UNSUPPORTED
    ctx2 = backends.make(backends.cuda(), cases.sod(32))
    with pytest.raises(abi.AbiError) as e:
        ctx2.adjoint_backward()
    assert e.value.status == abi.ERR_BAD_ARG


def test_vortex512_gradient_64_directions():
    """The adjoint workload as specified: 512^2 vortex to t = 2, checkpoint
    every 32 steps, gradient of J w.r.t. the initial (rho, rhoU, rhoV, E) on
    64 seeded unit-norm Gaussian directions, checked against
    - the forward-mode FP64 tangent: <= 1e-10 relative (same linearisation);
    - central differences in FP64 with the recorded dt sequence: <= 1e-6
      relative at h = 1e-6 or, where the FP64 noise of J(U0 +- h v) dominates
      that step (|<grad J, v>| ~ 1e-5 for unit directions over 1M values),
      at h = 1e-4."""
    n, t_end = 512, 2.0
    case = cases.vortex2d(n)
    ctx = backends.make(backends.cuda(), case)
    fids = cons_fids(2)
    U0 = torch.stack([torch.from_numpy(ctx.get_field(f).copy()) for f in fids])
    mask = torch.from_numpy(_interior_mask(ctx))
    x = case[1].x
    c = 0.5 * (x[:-1] + x[1:])
    X, Y = np.meshgrid(c, c, indexing="xy")
    disk = np.zeros(ctx.shape)
    ctx.interior(disk)[...] = ((X * X + Y * Y) < 1.0)[None] * (x[1] - x[0]) ** 2
    w = torch.from_numpy(disk)

    def J(U):
        return torch.sum(w * pressure(U) ** 2)

    U = U0.clone().requires_grad_(True)
    UN = SifvEvolve.apply(U, ctx, t_end, None, 32)
    sched = ctx.adjoint_schedule()
    J(UN).backward()
    grad = U.grad
    UNd = UN.detach().clone().requires_grad_(True)
    J(UNd).backward()
    gN = UNd.grad                      # dJ/dU(t_end) for the tangent check
    rng = np.random.default_rng(20261203)
    td_rel, fd6, fd_best = [], [], []
    for _ in range(64):
        v = torch.from_numpy(rng.standard_normal(U0.shape)) * mask
        v = v / torch.linalg.norm(v)
        ad = float(torch.sum(grad * v))
        for k, f in enumerate(fids):
            ctx.set_field(f, U0[k].numpy())
            ctx.tangent_set_direction(f, v[k].numpy())
        ctx.tangent_forward(0, 0.0, t_end, 0, sched)
        tv = torch.stack([torch.from_numpy(ctx.tangent_get(f).copy()) for f in fids])
        td_rel.append(abs(float(torch.sum(gN * tv)) - ad) / abs(ad))
        rel = []
        for h in (1e-6, 1e-4):
            with torch.no_grad():
                jp = J(SifvEvolve.apply(U0 + h * v, ctx, t_end, sched, 10 ** 6))
                jm = J(SifvEvolve.apply(U0 - h * v, ctx, t_end, sched, 10 ** 6))
            rel.append(abs(float((jp - jm) / (2 * h)) - ad) / abs(ad))
        fd6.append(rel[0])
        fd_best.append(min(rel))
    info = (max(td_rel), float(np.median(fd6)), max(fd6), max(fd_best))
    assert max(td_rel) <= 1e-10, info
    assert max(fd_best) <= 1e-6, info


def _gradient(case, t_end, lam, every, precision):
    ctx = backends.make(backends.cuda(), case)
    ctx.adjoint_set_precision(precision)
    ctx.adjoint_forward(0, 0.0, t_end, 0, every)
    for f, a in lam.items():
        ctx.adjoint_set_seed(f, a)
    ctx.adjoint_backward()
    return {f: ctx.adjoint_get_gradient(f) for f in lam}, ctx


@pytest.mark.parametrize("name", ["vortex", "riemann2d_walls", "sod"])
def test_fp32_reverse_sweep_close_to_fp64(name):
    """FP32 local Jacobians in the reverse sweep (the forward trajectory and
    the adjoint accumulation stay FP64): for random seeds the gradient
    agrees with the FP64 one to 1e-3 relative (L-infinity over the field's
    maximum; single-precision round-off accumulated over every stage)."""
    if name == "vortex":
        case, t_end = cases.vortex2d(64), 0.5
    elif name == "riemann2d_walls":
        case, t_end = cases.riemann2d(48, bc=abi.BC_SLIPWALL), 0.05
    else:
        case, t_end = cases.sod(200), 0.05
    probe = backends.make(backends.cuda(), case)
    rng = np.random.default_rng(11)
    mask = _interior_mask(probe)
    fids = cons_fids(case[0].dim)
    lam = {f: np.where(mask, rng.standard_normal(probe.shape), 0.0) for f in fids}
    g64, _ = _gradient(case, t_end, lam, 8, abi.PREC_FP64)
    g32, _ = _gradient(case, t_end, lam, 8, abi.PREC_MIXED)
    for f in fids:
        scale = np.abs(g64[f]).max()
        assert np.abs(g32[f] - g64[f]).max() <= 1e-3 * scale, f
        assert np.all(g32[f][~mask] == 0.0)


def test_fp32_reverse_sweep_rejects_other_precisions():
    ctx = backends.make(backends.cuda(), cases.sod(32))
    with pytest.raises(abi.AbiError) as e:
        ctx.adjoint_set_precision(abi.PREC_FP64_FAST)
    assert e.value.status == abi.ERR_BAD_ARG
