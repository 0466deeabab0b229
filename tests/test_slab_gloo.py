"""Slab decomposition of one problem over ranks, run on CPU: each gloo rank
steps its slab with the C oracle, exchanging ghost layers and reducing dt
through the library's hooks (sifv_set_comm, driven by
semiimplicitfv_b200.slab.DistExchange -- the same host code that drives
NCCL between GPUs).  The gathered result must equal the single-rank oracle
bit for bit: the explicit step exchanges only copies of cells and reduces
dt with an exact minimum, as the reference's MPI decomposition does."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import cases
from semiimplicitfv_b200 import abi

CASES = {
    "riemann2d-outflow-2": (lambda: cases.riemann2d(40), 2, 6),
    "riemann2d-periodic-ring-2": (lambda: cases.riemann2d(32, bc=abi.BC_PERIODIC), 2, 6),
    "riemann2d-slipwall-3": (lambda: cases.riemann2d(37, bc=abi.BC_SLIPWALL), 3, 6),
    "sod-1d-3": (lambda: cases.sod(150), 3, 20),
    "acoustic3d-periodic-2": (lambda: cases.acoustic3d(12, semi=False, igr=False, rk=3), 2, 3),
    "water-air-1d-2": (lambda: cases.water_air(96), 2, 10),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, out):
    import datetime
    import sys

    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import backends
    import cases as cs  # noqa: F401  (spawned process: the case builders)
    from semiimplicitfv_b200 import slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        make, _, nsteps = CASES[name]
        cfg, mesh, fields = make()
        lmesh, start, count = slab.slab_mesh(mesh, cfg.dim, rank, world)
        ax = slab.slab_axis(cfg.dim)
        periodic = mesh.bc[2 * ax] == abi.BC_PERIODIC
        ctx = backends.oracle().create(cfg, lmesh)
        ctx.set_state(slab.slab_fields(fields, cfg, start, count))
        slab.DistExchange(ctx, rank, world, periodic, device=False).attach()
        t, dts = 0.0, []
        for s in range(nsteps):
            dt = ctx.step(s, t, -1.0)
            dts.append(dt)
            t += dt
        out.put((rank, start, count, dts, {f: ctx.get_field(f) for f in fields}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", sorted(CASES))
def test_slab_decomposition_equals_single_rank(name):
    import backends
    make, world, nsteps = CASES[name]
    cfg, mesh, fields = make()
    single = backends.make(backends.oracle(), (cfg, mesh, fields))
    _, _, dts1 = cases.run_steps(single, nsteps)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from semiimplicitfv_b200 import slab
    glob = {f: np.zeros(single.shape) for f in fields}
    for rank, start, count, dts, loc in res:
        assert dts == dts1, (rank, dts, dts1)
        for f in fields:
            slab.gather_interior(loc[f], cfg, start, count, glob[f])
    for f in fields:
        a = single.interior(single.get_field(f))
        b = single.interior(glob[f])
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), (name, f, float(np.abs(a - b).max()))


def test_slab_split_matches_mpi_context():
    from semiimplicitfv_b200 import slab
    # MPIContext::sliceNodes: the first n % parts ranks take one more cell
    assert [slab.split(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    assert slab.neighbours(0, 3, False) == (None, 1)
    assert slab.neighbours(2, 3, True) == (1, 0)
    assert slab.neighbours(0, 2, True) == (1, 1)
