"""The semi-implicit step and IGR over a slab decomposition on the GPU.

Two ranks are emulated as two contexts on one GPU, each stepped by its own
host thread on its own stream; the halo exchange and the reductions (dt
minimum, pressure-residual maximum) go through the library's hooks as
stream-ordered device copies (no kernel waits on another).  The oracle runs
the same decomposition as two host contexts exchanging through the same
hooks; it is pinned to the reference's own MPI decomposition on CPU
(tests/test_slab_semi.py).  The gathered GPU result must equal the oracle's
bit for bit: fields, time steps and pressure iterations.  The IGR and
Gauss-Seidel sweeps run per rank in the reference's order (the tiled
wavefront and the 3D record sweeps included)."""
import threading

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi, slab
from test_gpu_slab import PairExchange

pytestmark = pytest.mark.gpu


class HostPair:
    """The hooks between two host (oracle) contexts stepped by two threads."""

    def __init__(self, ctxs, periodic):
        self.geo = [slab.DistExchange(c, r, 2, periodic, device=False) for r, c in enumerate(ctxs)]
        self.barrier = threading.Barrier(2, timeout=300)
        self.ptrs = [None, None]

    def hooks(self, r):
        g, peer = self.geo[r], 1 - r

        def exchange(ptrs, stream):
            self.ptrs[r] = ptrs
            self.barrier.wait()
            gp = self.geo[peer]
            for q, p in enumerate(ptrs):
                mine = slab._view(p, g.n, False)
                theirs = slab._view(self.ptrs[peer][q], gp.n, False)
                if g.lo is not None:
                    mine[g.low_ghost:g.low_ghost + g.block] = theirs[gp.high_int:gp.high_int + gp.block]
                if g.hi is not None:
                    mine[g.high_ghost:g.high_ghost + g.block] = theirs[gp.low_int:gp.low_int + gp.block]
            self.barrier.wait()   # both copies done before either rank writes its cells again
            return 0

        def reducer(op):
            def reduce(ptr, stream):
                self.ptrs[r] = ptr
                self.barrier.wait()
                v = op(slab._view(ptr, 1, False)[0].item(), slab._view(self.ptrs[peer], 1, False)[0].item())
                self.barrier.wait()   # both read before either writes
                slab._view(ptr, 1, False)[0] = v
                return 0
            return reduce
        return exchange, reducer(min), reducer(max)


def _explicit_igr_2d(n):
    cfg, mesh, fields = cases.riemann2d(n, riemann=abi.LF)
    cfg.useIGR, cfg.alphaCoeff, cfg.IGRIters, cfg.IGRWarmStartIters = 1, 10.0, 5, 20
    return cfg, mesh, fields


def _water_air_semi(n):
    cfg, mesh, fields = cases.water_air(n, p_left=2e5, rk=1)
    cfg.semiImplicit, cfg.siCfl, cfg.siMaxDt, cfg.pressureTol, cfg.maxPressureIters = 1, 0.5, 1e-4, 1e-6, 200
    return cfg, mesh, fields


# name: (case builder, steps, pressure solver 0 Jacobi / 1 Gauss-Seidel)
CASES = {
    "acoustic3d-semi-igr-jacobi": (lambda: cases.acoustic3d(16), 3, 0),
    "acoustic3d-semi-igr-gs": (lambda: cases.acoustic3d(32), 2, 1),
    "acoustic3d-semi-rk3-jacobi": (lambda: cases.acoustic3d(16, igr=False, rk=3), 2, 0),
    "box2d-semi-igr-slipwall": (lambda: cases.acoustic_box(48, 40, bc=abi.BC_SLIPWALL), 3, 0),
    "box2d-semi-igr-outflow-gs": (lambda: cases.acoustic_box(40, 41, bc=abi.BC_OUTFLOW), 2, 1),
    "advection1d-semi": (lambda: cases.advection1d(64, semi=True), 4, 0),
    "riemann2d-explicit-igr-lf": (lambda: _explicit_igr_2d(48), 3, 0),
    "water-air-semi": (lambda: _water_air_semi(96), 3, 0),
}


def _run_pair(backend, cfg, mesh, fields, nsteps, kind, device):
    ax = slab.slab_axis(cfg.dim)
    periodic = mesh.bc[2 * ax] == abi.BC_PERIODIC
    ctxs, parts = [], []
    for r in range(2):
        lmesh, start, count = slab.slab_mesh(mesh, cfg.dim, r, 2)
        c = backend.create(cfg, lmesh)
        c.set_state(slab.slab_fields(fields, cfg, start, count))
        if cfg.semiImplicit:
            c.set_pressure_solver(kind)
        ctxs.append(c)
        parts.append((start, count))
    pair = PairExchange(ctxs, periodic) if device else HostPair(ctxs, periodic)
    for r, c in enumerate(ctxs):
        c.set_comm(*pair.hooks(r))
    dts, iters, errors = [[], []], [[], []], []

    def run(r):
        try:
            t = 0.0
            for s in range(nsteps):
                dt = ctxs[r].step(s, t, -1.0)
                dts[r].append(dt)
                iters[r].append(ctxs[r].last_pressure_iterations() if cfg.semiImplicit else 0)
                t += dt
        except Exception as e:   # reported below; the barrier is aborted for the peer
            errors.append((r, repr(e)))
            pair.barrier.abort()
    threads = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=600)
    assert not errors, errors
    assert dts[0] == dts[1] and iters[0] == iters[1]
    shape = backends.make(backends.oracle(), (cfg, mesh, fields)).shape
    glob = {}
    for f in fields:
        glob[f] = np.zeros(shape)
        for c, (start, count) in zip(ctxs, parts):
            slab.gather_interior(c.get_field(f), cfg, start, count, glob[f])
    return dts[0], iters[0], glob


def _interior(cfg, arr):
    g = cfg.nGhost
    sl = [slice(None)] * 3
    for a in range(cfg.dim):
        sl[2 - a] = slice(g, arr.shape[2 - a] - g)
    return arr[tuple(sl)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_slabs_equal_oracle_slabs(name):
    make, nsteps, kind = CASES[name]
    cfg, mesh, fields = make()
    odts, oiters, oglob = _run_pair(backends.oracle(), cfg, mesh, fields, nsteps, kind, device=False)
    gdts, giters, gglob = _run_pair(backends.cuda(), cfg, mesh, fields, nsteps, kind, device=True)
    assert gdts == odts, (gdts, odts)
    assert giters == oiters, (giters, oiters)
    for f in fields:
        a, b = _interior(cfg, gglob[f]), _interior(cfg, oglob[f])
        assert np.all(np.isfinite(a)), (name, f)
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), (name, f, float(np.abs(a - b).max()))


def test_decomposed_pressure_solve_needs_the_max_reduction():
    cfg, mesh, fields = cases.acoustic3d(12)
    lmesh, start, count = slab.slab_mesh(mesh, 3, 0, 2)
    c = backends.cuda().create(cfg, lmesh)
    c.set_state(slab.slab_fields(fields, cfg, start, count))
    c.set_comm(lambda ptrs, stream: 0, lambda ptr, stream: 0)   # exchange and min only
    with pytest.raises(abi.AbiError) as e:
        c.step(0, 0.0, -1.0)
    assert e.value.status == abi.ERR_BAD_ARG
