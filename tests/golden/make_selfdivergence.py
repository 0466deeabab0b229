"""Measure how far the reference drifts from ITSELF when compiled with its
own Release flags (GCC's default FMA contraction) instead of
-ffp-contract=off, on the 2D four-quadrant Riemann problem (256^2, WENO5 +
HLLC, SSP-RK3, CFL 0.6) run to t = 0.8.  Writes
selfdivergence_riemann2d_256.json: per conserved variable the relative
L-infinity difference of the two builds.  Needs oracle/_ref (built from the
reference sources by oracle/Makefile); about 3 minutes of CPU."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import backends  # noqa: E402
import cases  # noqa: E402
from semiimplicitfv_b200 import abi  # noqa: E402


def main(n=256, t_end=0.8):
    a = backends.make(backends.reference(), cases.riemann2d(n))
    b = backends.make(backends.reference(release=True), cases.riemann2d(n))
    _, sa, _ = cases.run_steps(a, 10 ** 6, t_end)
    _, sb, _ = cases.run_steps(b, 10 ** 6, t_end)
    out = {"n": n, "t_end": t_end, "steps": [sa, sb], "rel_linf": {}}
    for name, fid in (("rho", abi.F_RHO), ("rhoU", abi.F_RHOU), ("rhoV", abi.F_RHOV), ("rhoE", abi.F_RHOE)):
        x, y = a.interior(a.get_field(fid)), b.interior(b.get_field(fid))
        out["rel_linf"][name] = float(np.abs(x - y).max() / np.abs(y).max())
    with open(os.path.join(HERE, f"selfdivergence_riemann2d_{n}.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
