"""Analytic pin: the oracle's Sod solution (config 1) converges to the exact
Riemann solution (Toro's exact solver) with the expected first-order L1
behaviour of a shock-capturing scheme."""
import numpy as np

import backends
import cases
import exact_riemann
from semiimplicitfv_b200 import abi


def sod_l1(backend, n, precision=abi.PREC_FP64):
    case = cases.sod(n)
    case[0].precision = precision
    c = backends.make(backend, case)
    cases.run_steps(c, 10 ** 6, t_end=0.2)
    x = 0.5 * (case[1].x[:-1] + case[1].x[1:])
    rho_e, _, _ = exact_riemann.sod_exact(x, 0.2)
    rho = c.interior(c.get_field(abi.F_RHO)).ravel()
    return np.abs(rho - rho_e).mean()


def test_exact_solver_star_state():
    p, u = exact_riemann.star_state(1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
    assert abs(p - 0.30313) < 1e-4 and abs(u - 0.92745) < 1e-4   # Toro, table 4.2, test 1


def test_oracle_sod_converges_to_exact():
    e = [sod_l1(backends.oracle(), n) for n in (100, 200, 400)]
    assert e[0] > e[1] > e[2]
    assert e[2] < 3e-3
    assert 0.5 < np.log2(e[1] / e[2]) < 1.5
