"""The fused-sweep paths on the GPU.

SIFV_PREC_FP64_FAST is FP64 with reassociated arithmetic: on the parity
cases it must stay within 1e-10 relative L-infinity per conserved variable
of the reference-ordered path (itself bit-identical to the reference); on a
long Kelvin-Helmholtz-unstable run it must drift no more than the reference
drifts from itself under its own Release compiler flags.  SIFV_PREC_MIXED runs the reconstruction / Riemann bulk in FP32:
it is judged by its L1 error against the exact solution (Sod) and against
the FP64 discretisation error."""
import json
import os

import numpy as np
import pytest

import backends
import cases
import exact_riemann
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu
TOL = 1e-10
CONS = (abi.F_RHO, abi.F_RHOU, abi.F_RHOE)


def _run(case, precision, nsteps, t_end=None, backend=None):
    case[0].precision = precision
    c = backends.make(backend or backends.cuda(), case)
    t, s, dts = cases.run_steps(c, nsteps, t_end)
    return c, dts


def _cons(cfg):
    f = list(CONS)
    if cfg.dim >= 2:
        f.append(abi.F_RHOV)
    if cfg.dim >= 3:
        f.append(abi.F_RHOW)
    return f


def _max_rel(ca, cb, cfg):
    worst = 0.0
    for fid in _cons(cfg):
        a, b = ca.interior(ca.get_field(fid)), cb.interior(cb.get_field(fid))
        worst = max(worst, np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    return worst


def test_fast_sod_full_config_vs_oracle():
    cf, dtf = _run(cases.sod(1000), abi.PREC_FP64_FAST, 10 ** 6, 0.2)
    co, dto = _run(cases.sod(1000), abi.PREC_FP64, 10 ** 6, 0.2, backends.oracle())
    assert len(dtf) == len(dto)
    assert _max_rel(cf, co, cf.cfg) <= TOL


@pytest.mark.parametrize("bc", [abi.BC_OUTFLOW, abi.BC_PERIODIC, abi.BC_SLIPWALL, abi.BC_NOSLIPWALL,
                                abi.BC_SYMMETRY])
@pytest.mark.parametrize("riemann", [abi.HLLC, abi.RUSANOV, abi.LF])
def test_fast_riemann2d(bc, riemann):
    cf, _ = _run(cases.riemann2d(48, bc=bc, riemann=riemann), abi.PREC_FP64_FAST, 20)
    co, _ = _run(cases.riemann2d(48, bc=bc, riemann=riemann), abi.PREC_FP64, 20, backend=backends.oracle())
    assert _max_rel(cf, co, cf.cfg) <= TOL


def test_fast_riemann2d_long_run_within_reference_self_divergence():
    """256^2 to t = 0.8 (the benchmark problem's full time at reduced size).
    The flow is Kelvin-Helmholtz unstable, so any change of rounding grows:
    the reference compiled with its own Release flags (FMA contraction)
    drifts from the same sources compiled without contraction by up to
    3.2e-9 relative L-inf per conserved variable on this run
    (golden/selfdivergence_riemann2d_256.json, made by
    golden/make_selfdivergence.py).  The fast-FP64 path must drift no more
    than that from the bit-exact path."""
    with open(os.path.join(os.path.dirname(__file__), "golden", "selfdivergence_riemann2d_256.json")) as f:
        bound = json.load(f)["rel_linf"]
    cf, dtf = _run(cases.riemann2d(256), abi.PREC_FP64_FAST, 10 ** 6, 0.8)
    ce, dte = _run(cases.riemann2d(256), abi.PREC_FP64, 10 ** 6, 0.8)
    assert len(dtf) == len(dte)
    for name, fid in (("rho", abi.F_RHO), ("rhoU", abi.F_RHOU), ("rhoV", abi.F_RHOV), ("rhoE", abi.F_RHOE)):
        a, b = cf.interior(cf.get_field(fid)), ce.interior(ce.get_field(fid))
        rel = np.abs(a - b).max() / np.abs(b).max()
        assert rel <= max(bound.values()), (name, rel, bound)


def test_fast_3d_explicit():
    case = lambda: cases.acoustic3d(16, semi=False, igr=False, rk=3)
    cf, _ = _run(case(), abi.PREC_FP64_FAST, 6)
    co, _ = _run(case(), abi.PREC_FP64, 6, backend=backends.oracle())
    assert _max_rel(cf, co, cf.cfg) <= TOL


def test_fast_stiffened_and_rk2():
    def case():
        c = cases.riemann2d(32, rk=2)
        c[0].eosKind = abi.EOS_STIFFENED
        c[0].pInf = 0.3
        return c
    cf, _ = _run(case(), abi.PREC_FP64_FAST, 10)
    co, _ = _run(case(), abi.PREC_FP64, 10, backend=backends.oracle())
    assert _max_rel(cf, co, cf.cfg) <= TOL


def test_fast_advance_matches_step():
    case = cases.riemann2d(64)
    case[0].precision = abi.PREC_FP64_FAST
    c1 = backends.make(backends.cuda(), case)
    c2 = backends.make(backends.cuda(), case)
    t1, s1, _ = cases.run_steps(c1, 9, t_end=0.05)
    t2, s2 = c2.advance(0, 0.0, 0.05, 9)
    assert (t1, s1) == (t2, s2)
    for fid in _cons(case[0]):
        assert np.array_equal(c1.get_field(fid), c2.get_field(fid))


def test_unsupported_configs_rejected():
    case = cases.water_air(32)
    case[0].precision = abi.PREC_MIXED
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(case[0], case[1])
    assert e.value.status == abi.ERR_UNSUPPORTED


def _sod_l1(precision, n):
    case = cases.sod(n)
    c, _ = _run(case, precision, 10 ** 6, 0.2)
    x = 0.5 * (case[1].x[:-1] + case[1].x[1:])
    rho_e, _, _ = exact_riemann.sod_exact(x, 0.2)
    return np.abs(c.interior(c.get_field(abi.F_RHO)).ravel() - rho_e).mean()


@pytest.mark.parametrize("n", [1000, 4000])
def test_mixed_sod_error_within_bound(n):
    """Mixed-precision L1 error against the exact solution within 1.5x of the
    FP64 discretisation error."""
    e64 = _sod_l1(abi.PREC_FP64, n)
    emx = _sod_l1(abi.PREC_MIXED, n)
    assert emx <= 1.5 * e64, (emx, e64)


def test_mixed_riemann2d_error_within_bound():
    """2D Riemann 256^2 to t = 0.25: the mixed-vs-FP64 difference is well
    below the FP64 discretisation error (FP64 256^2 vs FP64 512^2 averaged
    onto 256^2)."""
    t_end = 0.25
    c64, _ = _run(cases.riemann2d(256), abi.PREC_FP64_FAST, 10 ** 6, t_end)
    cmx, _ = _run(cases.riemann2d(256), abi.PREC_MIXED, 10 ** 6, t_end)
    cfine, _ = _run(cases.riemann2d(512), abi.PREC_FP64_FAST, 10 ** 6, t_end)
    r64 = c64.interior(c64.get_field(abi.F_RHO))[0]
    rmx = cmx.interior(cmx.get_field(abi.F_RHO))[0]
    rf = cfine.interior(cfine.get_field(abi.F_RHO))[0]
    rf = 0.25 * (rf[0::2, 0::2] + rf[1::2, 0::2] + rf[0::2, 1::2] + rf[1::2, 1::2])
    disc = np.abs(r64 - rf).mean()
    mixed_vs_fp64 = np.abs(rmx - r64).mean()
    err_mx = np.abs(rmx - rf).mean()
    assert err_mx <= 1.5 * disc, (err_mx, disc)
    assert mixed_vs_fp64 < 0.1 * disc, (mixed_vs_fp64, disc)


def test_fast_reciprocal_and_sqrt_within_one_ulp():
    """The fast paths' refined reciprocal, square root and reciprocal square
    root against IEEE 1/x, sqrt(x) and 1/sqrt(x) on 2^22 arguments across
    [2^-60, 2^60): within one ulp (2^-52 relative; the reference 1/sqrt(x)
    is itself rounded twice, so that bound gets half an ulp more)."""
    import ctypes
    from semiimplicitfv_b200 import _lib
    lib = _lib.load()
    lib.sifv_fastmath_selftest.argtypes = [ctypes.c_longlong] + [ctypes.POINTER(ctypes.c_double)] * 3
    r, s, q = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    assert lib.sifv_fastmath_selftest(1 << 22, ctypes.byref(r), ctypes.byref(s), ctypes.byref(q)) == 0
    assert r.value <= 2.23e-16, r.value
    assert s.value <= 2.23e-16, s.value
    assert q.value <= 3.34e-16, q.value


@pytest.mark.parametrize("prec", [abi.PREC_FP64_FAST, abi.PREC_MIXED])
def test_autotuned_work_units_leave_results_unchanged(prec):
    """sifv_autotune picks the work-unit shape of the fused 2D stage by
    timing; every shape computes each cell with the same arithmetic, so the
    state after the same steps is bit-identical, and the probe launches do
    not touch the state."""
    def run(units):
        case = cases.riemann2d(300)
        case[0].precision = prec
        c = backends.make(backends.cuda(), case)
        chosen = None
        if units == "tune":
            chosen = c.autotune(3)
        elif units is not None:
            c.set_work_units(units)
        cases.run_steps(c, 6)
        return c, chosen
    a, _ = run(None)
    b, chosen = run("tune")
    assert chosen in (1, 2, 3, 4)
    runs = [b] + [run(u)[0] for u in (1, 2, 3, 4)]
    for fid in (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE, abi.F_PRES):
        x = a.get_field(fid)
        for r in runs:
            assert np.array_equal(x.view(np.int64), r.get_field(fid).view(np.int64)), fid
    with pytest.raises(abi.AbiError):
        a.set_work_units(5)
