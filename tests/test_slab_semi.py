"""The semi-implicit step and IGR over a slab decomposition, on CPU.

Each gloo rank steps its slab with the C oracle through the library's hooks
(sifv_set_comm, driven by semiimplicitfv_b200.slab.DistExchange); the
reference's own solver runs the same decomposition (MPIContext::create with
one rank per slab along the slowest axis, ranks as threads through the MPI
shim).  The IGR and Gauss-Seidel sweeps run over each rank's own cells in
the reference's order with the neighbour's values from the last exchange
(src/IGR.cpp:110-156, src/GaussSeidelPressureSolver.cpp:54-103), so the
decomposed run is a different iteration from the single-domain one: the
oracle must equal the decomposed reference bit for bit, fields, time steps
and pressure iterations.  (Even without IGR the decomposed semi-implicit
step is not the single-domain one in the last bits: each rank derives the
ghost-cell widths at its cuts from its own nodes, as the reference's local
RectilinearMesh does, and the pressure Laplacian's face distances use
them.)  No GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import backends
import cases
from semiimplicitfv_b200 import abi


def _ref():
    ref = backends.reference()
    if ref is None:
        pytest.skip("reference build absent (oracle/_ref)")
    return ref


def _explicit_igr_2d():
    cfg, mesh, fields = cases.riemann2d(32, riemann=abi.LF)
    cfg.useIGR, cfg.alphaCoeff, cfg.IGRIters, cfg.IGRWarmStartIters = 1, 10.0, 5, 20
    return cfg, mesh, fields


def _water_air_semi():
    cfg, mesh, fields = cases.water_air(72, p_left=2e5, rk=1)
    cfg.semiImplicit, cfg.siCfl, cfg.siMaxDt, cfg.pressureTol, cfg.maxPressureIters = 1, 0.5, 1e-4, 1e-6, 200
    return cfg, mesh, fields


# name: (case builder, ranks, steps, pressure solver 0 Jacobi / 1 Gauss-Seidel)
CASES = {
    "acoustic3d-semi-igr-jacobi-2": (lambda: cases.acoustic3d(12), 2, 3, 0),
    "acoustic3d-semi-igr-gs-3": (lambda: cases.acoustic3d(12), 3, 2, 1),
    "acoustic3d-semi-rk2-jacobi-2": (lambda: cases.acoustic3d(12, igr=False, rk=2), 2, 2, 0),
    "box2d-semi-igr-slipwall-2": (lambda: cases.acoustic_box(24, 20, bc=abi.BC_SLIPWALL), 2, 3, 0),
    "box2d-semi-igr-outflow-gs-3": (lambda: cases.acoustic_box(20, 21, bc=abi.BC_OUTFLOW), 3, 2, 1),
    "advection1d-semi-3": (lambda: cases.advection1d(60, semi=True), 3, 4, 0),
    "riemann2d-explicit-igr-lf-2": (_explicit_igr_2d, 2, 3, 0),
    "water-air-semi-2": (_water_air_semi, 2, 3, 0),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _procs(dim, ranks):
    return {1: (ranks, 1, 1), 2: (1, ranks, 1), 3: (1, 1, ranks)}[dim]


def _worker(rank, world, port, name, out):
    import datetime
    import sys

    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import backends as be
    from semiimplicitfv_b200 import slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        make, _, nsteps, kind = CASES[name]
        cfg, mesh, fields = make()
        lmesh, start, count = slab.slab_mesh(mesh, cfg.dim, rank, world)
        ax = slab.slab_axis(cfg.dim)
        periodic = mesh.bc[2 * ax] == abi.BC_PERIODIC
        ctx = be.oracle().create(cfg, lmesh)
        ctx.set_state(slab.slab_fields(fields, cfg, start, count))
        if cfg.semiImplicit:
            ctx.set_pressure_solver(kind)
        slab.DistExchange(ctx, rank, world, periodic, device=False).attach()
        t, dts, iters = 0.0, [], []
        for s in range(nsteps):
            dt = ctx.step(s, t, -1.0)
            dts.append(dt)
            iters.append(ctx.last_pressure_iterations() if cfg.semiImplicit else 0)
            t += dt
        out.put((rank, start, count, dts, iters, {f: ctx.get_field(f) for f in fields}))
    finally:
        dist.destroy_process_group()


def _run_oracle_slabs(name):
    make, world, _, _ = CASES[name]
    cfg, mesh, fields = make()
    shape = backends.make(backends.oracle(), (cfg, mesh, fields)).shape
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from semiimplicitfv_b200 import slab
    glob = {f: np.zeros(shape) for f in fields}
    dts = iters = None
    for rank, start, count, d, it, loc in res:
        if dts is None:
            dts, iters = d, it
        assert d == dts and it == iters, (rank, d, dts)
        for f in fields:
            slab.gather_interior(loc[f], cfg, start, count, glob[f])
    return dts, iters, glob


def _interior(cfg, arr):
    g = cfg.nGhost
    sl = [slice(None)] * 3
    for a in range(cfg.dim):
        sl[2 - a] = slice(g, arr.shape[2 - a] - g)
    return arr[tuple(sl)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_slabs_equal_decomposed_reference(name):
    ref = _ref()
    make, world, nsteps, kind = CASES[name]
    cfg, mesh, fields = make()
    dts, iters, glob = _run_oracle_slabs(name)
    _, rdts, dims, rfields, riters = backends.mpi_run(ref, (cfg, mesh, fields), world, 0, nsteps,
                                                      procs=_procs(cfg.dim, world), pressure_kind=kind)
    assert dims == _procs(cfg.dim, world)
    assert dts == rdts, (dts, rdts)
    if cfg.semiImplicit:
        assert iters == riters, (iters, riters)
    for f in fields:
        a, b = _interior(cfg, glob[f]), _interior(cfg, rfields[f].reshape(glob[f].shape))
        assert np.all(np.isfinite(a)), (name, f)
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), (name, f, float(np.abs(a - b).max()))
