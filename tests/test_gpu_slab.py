"""Slab decomposition on the GPU: two ranks emulated as two contexts on one
GPU, each stepped by its own host thread on its own stream.  The halo
exchange and the dt reduction go through the library's hooks
(sifv_set_comm) as in a multi-GPU run; here they are device-to-device
copies ordered with CUDA events between the two streams (no kernel waits on
another: every dependency is a stream-event wait).  The gathered result must
equal the single-context run bit for bit, for the reference-ordered FP64
step (1D, 2D, 3D) and the fast / mixed 2D step."""
import threading

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi, slab

pytestmark = pytest.mark.gpu


class PairExchange:
    """Halo exchange and dt minimum between two contexts of one process."""

    def __init__(self, ctxs, periodic):
        import torch
        self.ctxs = ctxs
        self.geo = [slab.DistExchange(c, r, 2, periodic, device=True) for r, c in enumerate(ctxs)]
        self.streams = [torch.cuda.Stream() for _ in ctxs]
        for c, s in zip(ctxs, self.streams):
            c.be.fn["set_stream"](c.h, s.cuda_stream)
        self.barrier = threading.Barrier(2, timeout=120)
        self.ready = [torch.cuda.Event() for _ in ctxs]
        self.copied = [torch.cuda.Event() for _ in ctxs]
        self.ptrs = [None, None]
        self.tmp = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in ctxs]

    def _sync(self, r, body):
        import torch
        peer = 1 - r
        s = self.streams[r]
        self.ready[r].record(s)
        self.barrier.wait()
        s.wait_event(self.ready[peer])
        with torch.cuda.stream(s):
            body(peer)
        self.copied[r].record(s)
        self.barrier.wait()
        s.wait_event(self.copied[peer])

    def hooks(self, r):
        g = self.geo[r]

        def exchange(ptrs, stream):
            self.ptrs[r] = ptrs

            def body(peer):
                gp = self.geo[peer]
                for q, p in enumerate(ptrs):
                    mine = slab._view(p, g.n, True)
                    theirs = slab._view(self.ptrs[peer][q], gp.n, True)
                    if g.lo is not None:
                        mine[g.low_ghost:g.low_ghost + g.block].copy_(theirs[gp.high_int:gp.high_int + gp.block])
                    if g.hi is not None:
                        mine[g.high_ghost:g.high_ghost + g.block].copy_(theirs[gp.low_int:gp.low_int + gp.block])
            self._sync(r, body)
            return 0

        def reducer(op):
            def reduce(ptr, stream):
                import torch
                self.ptrs[r] = ptr
                self._sync(r, lambda peer: self.tmp[r].copy_(slab._view(self.ptrs[peer], 1, True)))
                with torch.cuda.stream(self.streams[r]):
                    v = slab._view(ptr, 1, True)
                    op(v, self.tmp[r], out=v)
                self.barrier.wait()   # both results taken before either rank reuses its pointer slot
                return 0
            return reduce
        import torch
        return exchange, reducer(torch.minimum), reducer(torch.maximum)


CASES = {
    "riemann2d-fp64": (lambda: cases.riemann2d(64), abi.PREC_FP64, 6),
    "riemann2d-periodic-fast": (lambda: cases.riemann2d(64, bc=abi.BC_PERIODIC), abi.PREC_FP64_FAST, 8),
    "riemann2d-mixed": (lambda: cases.riemann2d(96), abi.PREC_MIXED, 8),
    "riemann2d-slipwall-fast-rk2": (lambda: cases.riemann2d(70, bc=abi.BC_SLIPWALL, rk=2), abi.PREC_FP64_FAST, 8),
    "sod-1d-fp64": (lambda: cases.sod(200), abi.PREC_FP64, 20),
    "acoustic3d-periodic-fp64": (lambda: cases.acoustic3d(16, semi=False, igr=False, rk=3), abi.PREC_FP64, 3),
    "water-air-1d-fp64": (lambda: cases.water_air(128), abi.PREC_FP64, 10),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_slab_contexts_equal_one(name):
    make, prec, nsteps = CASES[name]
    cfg, mesh, fields = make()
    cfg.precision = prec
    single = backends.make(backends.cuda(), (cfg, mesh, fields))
    _, _, dts1 = cases.run_steps(single, nsteps)
    ax = slab.slab_axis(cfg.dim)
    periodic = mesh.bc[2 * ax] == abi.BC_PERIODIC
    ctxs, parts = [], []
    for r in range(2):
        lmesh, start, count = slab.slab_mesh(mesh, cfg.dim, r, 2)
        c = backends.cuda().create(cfg, lmesh)
        c.set_state(slab.slab_fields(fields, cfg, start, count))
        ctxs.append(c)
        parts.append((start, count))
    pair = PairExchange(ctxs, periodic)
    for r, c in enumerate(ctxs):
        c.set_comm(*pair.hooks(r))
    dts = [[], []]
    errors = []

    def run(r):
        try:
            t = 0.0
            for s in range(nsteps):
                dt = ctxs[r].step(s, t, -1.0)
                dts[r].append(dt)
                t += dt
        except Exception as e:   # reported below; the barrier timeout ends the peer
            errors.append((r, repr(e)))
            pair.barrier.abort()
    threads = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not errors, errors
    assert dts[0] == dts1 and dts[1] == dts1, (dts, dts1)
    for f in fields:
        glob = np.zeros(single.shape)
        for c, (start, count) in zip(ctxs, parts):
            slab.gather_interior(c.get_field(f), cfg, start, count, glob)
        a, b = single.interior(single.get_field(f)), single.interior(glob)
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), (name, f, float(np.abs(a - b).max()))


def test_exchange_faces_need_the_hooks():
    cfg, mesh, fields = cases.riemann2d(32)
    lmesh, start, count = slab.slab_mesh(mesh, 2, 0, 2)
    c = backends.cuda().create(cfg, lmesh)
    c.set_state(slab.slab_fields(fields, cfg, start, count))
    with pytest.raises(abi.AbiError) as e:
        c.step(0, 0.0, -1.0)
    assert e.value.status == abi.ERR_BAD_ARG


def test_exchange_faces_reject_unsupported_configs():
    cfg, mesh, _ = cases.acoustic3d(12)   # semi-implicit + IGR, mixed precision (FP32 Jacobi sweeps)
    cfg.precision = abi.PREC_MIXED
    lmesh, _, _ = slab.slab_mesh(mesh, 3, 0, 2)
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(cfg, lmesh)
    assert e.value.status == abi.ERR_UNSUPPORTED
    cfg, mesh, _ = cases.riemann2d(32)
    cfg.mu = 1e-3                          # viscous fluxes
    lmesh, _, _ = slab.slab_mesh(mesh, 2, 0, 2)
    with pytest.raises(abi.AbiError) as e:
        backends.cuda().create(cfg, lmesh)
    assert e.value.status == abi.ERR_UNSUPPORTED
