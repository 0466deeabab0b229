"""Benchmark: cell-updates/s of the SSP-RK3 WENO5-HLLC step on the 2D
four-quadrant Riemann problem, 4096 x 4096 cells, FP64.

One "step" is one full time step (three RK stages, dt reduction, ghost
fills) over the whole grid.  `value` times K steps queued back to back with
the state resident in HBM (sifv_advance); `e2e` times K steps the way the
drop-in solver with host-authoritative state runs them: per step the state
fields the step reads are copied from pinned host buffers (sifv_set_field),
sifv_step runs and returns dt, and the fields it writes are copied back
(sifv_get_field).  The same JSON line carries the other workloads as
objects: `semi_implicit` (3D acoustic pulse 256^3 with IGR and the Jacobi
pressure solve), `semi_implicit_2d_periodic` (2D 2048^2 periodic with IGR
and the Gauss-Seidel pressure solve, the 2D wavefront kernels against the
tiled sweeps), `adjoint` (isentropic-vortex discrete adjoint 512^2) and
`ensemble` (2048 two-phase water-air tubes in one launch).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

Multi-GPU: one process per GPU (torchrun); the 4096^2 grid is cut into
slabs of rows, one per rank, with the 3-row halo exchange of every RK stage
and the dt all-reduce over NCCL (strong scaling); time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "cell-updates/s per RK3 step (2D Riemann 4096^2, WENO5+HLLC, FP64)"
PREC_NAMES = {0: "fp64-reference-order", 1: "mixed-fp32-bulk", 2: "fp64-fast"}
UNIT = "cell-updates/s"
BYTES_PER_CELL_UPDATE = 256   # algorithmic: 64 B x 4 conserved variables per RK3 step
# Algorithmic bytes per cell of one launch of each kernel family of the 2D
# step (FP64 arrays, 8 B per value):
#   march2d  one fused kernel per stage: reads U (4) and, in stages 2-3, U0
#            (4); writes U' (4); the last stage also writes u, v, p (3)
#                                             (32 + 21.33 + 32 + 8) = 93.33
#   dt       reads rho, velU, velV, pres                         4 x 8 = 32
#   bc_prim  ghost cells only (negligible per interior cell)
KERNEL_BYTES_PER_CELL_2D = {"march2d": 93.33, "dt": 32.0, "bc_prim": 0.0, "face_x": 64.0, "face_y": 64.0,
                            "assemble": 229.3, "prim_bc": 56.0}
# Per launch of the dominant kernel, measured by ncu on the 2048^2 case of the
# same workload (3 launches = one step, averaged): DRAM bytes per cell
# (dram__bytes_read.sum + dram__bytes_write.sum) and FP64 / FMA-pipe
# instructions per cell, with the SHA-1 of the kernel sources they were taken
# on.  When the sources have changed since, the figures are reported as stale
# (traffic null) instead of being applied to a different kernel.
NCU_KERNEL_SOURCES = ("semiimplicitfv_b200/csrc/sifv_march2d.cuh", "semiimplicitfv_b200/csrc/sifv_sweep.cuh",
                      "semiimplicitfv_b200/csrc/sifv_fastmath.cuh")
# (precision, kernel) -> {"sha": ..., "dram_bytes_per_cell": ..., "fp64_inst_per_cell": ...}; from
# one ncu capture each of the FP64 and the mixed march kernel on a 2048² four-quadrant Riemann stage
# (FP64 thread operations: DADD + DMUL + DFMA issued, per interior cell)
NCU_CAPTURE = {
    (2, "march2d"): {"sha": "32a04e8cb0599297", "dram_bytes_per_cell": 89.50, "fp64_inst_per_cell": 838.1},
    (1, "march2d"): {"sha": "32a04e8cb0599297", "dram_bytes_per_cell": 94.32, "fp64_inst_per_cell": 46.4},
}


def _kernel_sources_sha() -> str:
    import hashlib
    h = hashlib.sha1()
    for f in NCU_KERNEL_SOURCES:
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


# Fields a 2D step reads and writes (host-authoritative drop-in round trip).
E2E_FIELDS_2D = ("F_RHO", "F_RHOU", "F_RHOV", "F_RHOE", "F_VELU", "F_VELV", "F_PRES")
CONS_NAMES_2D = ("rho", "rhoU", "rhoV", "rhoE")
# Batched ensemble of two-phase water-air tubes: count, cell range, end time.
ENS_COUNT, ENS_NMIN, ENS_NMAX, ENS_TEND, ENS_SEED = 2048, 256, 16384, 1e-4, 0
ENS_BYTES_PER_CELL_UPDATE = 384   # state alphaRho0, alphaRho1, rhoU, rhoE, alpha0, alpha1: 64 B x 6
# Semi-implicit 3D acoustic pulse with IGR, 256^3 periodic, RK1: 20 timed steps.
# Algorithmic bytes per cell-update: 272 + 32 per IGR sweep + 40 per Jacobi iteration.
SI_N, SI_STEPS, SI_WARM = 256, 20, 3
SI2_N, SI2_STEPS = 2048, 3          # the 2D periodic semi-implicit steps (wavefront vs tiles)
# Discrete adjoint: isentropic vortex 512^2 to t = 2, checkpoint every 32 steps.
# Algorithmic bytes per adjoint cell-update: forward recompute 256 + store and
# read the three stage states 2 x 96 + adjoint state read/write per stage 3 x 64.
ADJ_N, ADJ_TEND, ADJ_EVERY, ADJ_BYTES_PER_CELL_UPDATE = 512, 2.0, 32, 640
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")


def _peaks():
    try:
        with open(PEAKS_FILE) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []          # (host time, csv line)
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:   # wait for the sampler to run
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t_start: float, t_end: float):
        self.window = (t_start, t_end)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if self.window:   # samples taken while the timed region ran (0.1 s slack for pipe latency)
            inside = [x for x in lines if self.window[0] - 0.1 <= x[0] <= self.window[1] + 0.1]
            lines = inside or lines
        for _, ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ensemble_instances(count=ENS_COUNT, seed=ENS_SEED, nmin=ENS_NMIN, nmax=ENS_NMAX):
    """Seeded two-phase water-air tubes on [0, 1]: cells log-uniform in
    [nmin, nmax], interface uniform in [0.3, 0.7], water pressure uniform in
    [1e8, 1e9] (water gamma 4.4, pInf 6e8, rho 1000; air gamma 1.4, rho 1,
    p 1e5; alphaMin 1e-8), WENO5 + mixture HLLC, SSP-RK3, CFL 0.5."""
    import numpy as np
    import cases
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(np.log(nmin), np.log(nmax), count))).astype(int)
    xi = rng.uniform(0.3, 0.7, count)
    pl = rng.uniform(1e8, 1e9, count)
    return [cases.water_air(int(n), x_interface=float(a), p_left=float(b)) for n, a, b in zip(ns, xi, pl)]


def _ens_cpu_worker(args):
    """One process: the reference (or oracle) runs its share of tubes alone,
    each to the end time; returns (cell-updates, seconds)."""
    kind, idx = args
    import backends
    import cases
    be = backends.reference(release=True) if kind == "reference" else backends.oracle()
    inst = ensemble_instances()
    cu, sec = 0.0, 0.0
    for k in idx:
        case = inst[k]
        ctx = backends.make(be, case)
        t0 = time.perf_counter()
        _, steps, _ = cases.run_steps(ctx, 10 ** 9, t_end=ENS_TEND)
        sec += time.perf_counter() - t0
        cu += (len(case[1].x) - 1) * steps
    return cu, sec


def ensemble_cpu_rate(kind, procs, budget_cells=1500):
    """Aggregate cell-updates/s of `procs` concurrent single-thread processes,
    each running seeded tubes of the ensemble whose cell count is at most
    `budget_cells` (a bounded sample: cost per cell-update does not depend
    on the tube length)."""
    inst = ensemble_instances()
    small = [k for k, c in enumerate(inst) if len(c[1].x) - 1 <= budget_cells]
    per = max(1, min(len(small) // max(procs, 1), 4))
    shares = [small[(p * per) % len(small):(p * per) % len(small) + per] for p in range(procs)]
    with mp.get_context("spawn").Pool(procs) as pool:
        out = pool.map(_ens_cpu_worker, [(kind, sh) for sh in shares])
    rate = sum(cu / sec for cu, sec in out if sec > 0)
    return rate, f"{procs} concurrent single-thread processes x {per} seeded tubes of <= {budget_cells} cells each"


def semi_cpu_rate(kind, n=64, steps=2):
    """Reference (or oracle) semi-implicit 3D step on one core: an n^3
    instance of the same problem, `steps` steps after step 0 (the IGR warm
    start).  Fewer Jacobi iterations than at 256^3 (they grow with n), so
    this overstates the CPU rate per cell at the full size."""
    import backends
    import cases
    be = backends.reference(release=True) if kind == "reference" else backends.oracle()
    ctx = backends.make(be, cases.acoustic3d(n))
    t = ctx.step(0, 0.0, -1.0)
    t0 = time.perf_counter()
    for s in range(steps):
        t += ctx.step(1 + s, t, -1.0)
    sec = time.perf_counter() - t0
    return n ** 3 * steps / sec, f"{n}^3 instance, {steps} steps after the warm-start step, 1 thread"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_rate(kind: str, n: int, steps: int) -> float:
    """Reference (or oracle) CPU path on one core: cell-updates/s on an n x n
    instance of the same problem, `steps` steps after one warm-up step."""
    import backends
    import cases
    be = backends.reference(release=True) if kind == "reference" else backends.oracle()
    ctx = backends.make(be, cases.riemann2d(n))
    ctx.step(0, 0.0, -1.0)
    t0 = time.perf_counter()
    t = 0.0
    for s in range(steps):
        t += ctx.step(1 + s, t, -1.0)
    dt = time.perf_counter() - t0
    return n * n * steps / dt


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def workload_config(n: int) -> dict:
    """The `config` object both arms print (the same workload)."""
    return {"workload": f"2D four-quadrant Riemann {n}x{n} (+3 ghosts), WENO5+HLLC SSP-RK3 CFL0.6, outflow",
            "l2": (f"inputs larger than L2 (state 4 x {n * n * 8 / 1e6:.0f} MB)" if 4 * n * n * 8 > 126e6
                   else f"state 4 x {n * n * 8 / 1e6:.0f} MB fits in L2")}


def reference_decomposed_rate(n: int, warmup: int, steps: int, ranks: int):
    """The reference's own solver on the n x n workload, decomposed over
    `ranks` MPI ranks (threads through the MPI shim; the reference is
    single-threaded per rank): `warmup` steps, then `steps` timed steps.
    Returns (cell-updates/s, seconds, process grid)."""
    import backends
    import cases
    be = backends.reference(release=True)
    sec, _, dims, _, _ = backends.mpi_run(be, cases.riemann2d(n), ranks, warmup, steps, gather=False)
    return n * n * steps / sec, sec, dims


def run_reference(args):
    """--impl reference: the reference's CPU solver on the same 4096^2
    workload, all host cores (one MPI rank per core through the MPI shim,
    the reference's own domain decomposition and halo exchange), W warm-up
    steps then K timed steps of the full grid."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    import backends
    n = args.n
    cores = _host_cores()
    if backends.reference(release=True) is not None:
        value, sec, dims = reference_decomposed_rate(n, args.warmup, args.steps, cores)
        kind = "reference"
        sample = (f"{n}x{n}, {args.warmup} warm-up + {args.steps} timed steps of the full grid, decomposed over "
                  f"{cores} MPI ranks ({dims[0]}x{dims[1]}; threads of one process through the MPI shim), "
                  f"reference built with its Release flags; wall {sec:.1f} s for the timed steps")
    else:   # the reference sources were never built here: the oracle port on one core, bounded sample
        value = cpu_rate("port", 768, 3)
        sec = n * n * args.steps / value
        kind, cores = "port", 1
        sample = "C restatement on one core, 768x768 instance, 3 steps (reference build absent)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "precision": "fp64 (the reference's CPU solver)",
        "config": workload_config(n),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_cuda(args):
    import numpy as np
    import torch

    ws, rank, local = _dist()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)

    import backends
    import cases
    from semiimplicitfv_b200 import abi, slab
    CONS_2D = (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE)
    n = args.n
    cells = n * n
    stream = torch.cuda.current_stream()

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    def max_over_ranks(x: float) -> float:
        if ws > 1:
            t = torch.tensor([x], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            return float(t.item())
        return x

    def make_ctx(precision):
        """This rank's context: the whole grid on one GPU; with N ranks its
        slab of rows (slab decomposition along y, halo exchange and dt
        reduction over NCCL through the library's hooks)."""
        case = cases.riemann2d(n)
        case[0].precision = precision
        mesh, fields = case[1], case[2]
        if ws > 1:
            mesh, start, count = slab.slab_mesh(case[1], 2, rank, ws)
            fields = slab.slab_fields(case[2], case[0], start, count)
        ctx = backends.cuda().create(case[0], mesh, local)
        for fid, arr in fields.items():   # inputs uploaded from pinned host memory
            pinned = torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
            ctx.be.fn["set_field"](ctx.h, fid, ctypes.c_void_p(pinned.data_ptr()), 0)
        ctx.be.fn["set_stream"](ctx.h, ctypes.c_void_p(stream.cuda_stream))
        if ws > 1:
            slab.DistExchange(ctx, rank, ws, periodic=False, device=True).attach()
        if args.units_per_warp:
            ctx.set_work_units(args.units_per_warp)
            ctx.tuned = args.units_per_warp
        else:
            ctx.tuned = ctx.autotune(5)   # work-unit shape of the fused stage kernel (part of the warm-up)
        return ctx

    def measure(precision, with_clocks=False, with_e2e=False):
        ctx = make_ctx(precision)
        clk = ClockSampler(local) if with_clocks else None
        if clk:
            clk.__enter__()
        t_sim, _ = ctx.advance(0, 0.0, -1.0, args.warmup)
        step_idx = args.warmup
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.time()
        e0.record(stream)
        t_sim, _ = ctx.advance(step_idx, t_sim, -1.0, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.mark(w0, time.time())
            clk.__exit__(None, None, None)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        step_idx += args.steps
        _, launches = ctx.last_step_stats()
        out = {"ms": ms, "value": cells * args.steps / (ms / 1e3), "launches": launches, "tuned": ctx.tuned,
               "clocks": clk.summary() if clk else None, "t": t_sim,
               # the conservative state after the warm-up and timed steps (error against FP64)
               "state": {f: ctx.interior(ctx.get_field(f)).copy() for f in CONS_2D} if ws == 1 else None}
        if with_clocks:
            # per-kernel-family device time of two more steps (CUDA events on the launch stream)
            fam = {}
            for q in range(2):
                for k, (fms, cnt) in ctx.profile_step(step_idx + q, t_sim, -1.0).items():
                    a = fam.setdefault(k, [0.0, 0])
                    a[0] += fms
                    a[1] += cnt
            step_idx += 2
            out["families"] = fam
        if with_e2e:
            # (1) device-resident drop-in (state stays on the GPU, dt back to the host each step)
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            for q in range(args.steps):
                t_sim += ctx.step(step_idx + q, t_sim, -1.0)
            torch.cuda.synchronize()
            out["e2e_resident"] = cells * args.steps / max_over_ranks(time.perf_counter() - t0)
            step_idx += args.steps
            # (2) host-authoritative drop-in: per step the fields the step reads go up
            # from pinned host buffers, sifv_step runs, the fields it writes come back
            fids = [getattr(abi, f) for f in E2E_FIELDS_2D]
            host = {f: torch.from_numpy(ctx.get_field(f).reshape(-1).copy()).pin_memory() for f in fids}
            set_f, get_f, step_f = ctx.be.fn["set_field"], ctx.be.fn["get_field"], ctx.be.fn["step"]
            dtv = ctypes.c_double()
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            for q in range(args.steps):
                for f in fids:
                    assert set_f(ctx.h, f, ctypes.c_void_p(host[f].data_ptr()), 0) == 0
                assert step_f(ctx.h, step_idx + q, t_sim, -1.0, ctypes.byref(dtv)) == 0
                t_sim += dtv.value
                for f in fids:
                    assert get_f(ctx.h, f, ctypes.c_void_p(host[f].data_ptr()), 0) == 0
            torch.cuda.synchronize()
            out["e2e"] = cells * args.steps / max_over_ranks(time.perf_counter() - t0)
            out["e2e_bytes"] = len(fids) * ctx.ncells * 8
        ctx.close()
        return out

    def measure_fine(t_final):
        """The same problem on a 2n x 2n grid, reference-ordered FP64, run
        to t_final, averaged over 2 x 2 blocks onto the n x n cells (exact
        restriction of finite-volume cell averages): the reference solution
        of the discretisation error."""
        case = cases.riemann2d(2 * n)
        case[0].precision = abi.PREC_FP64
        ctx = backends.cuda().create(case[0], case[1], local)
        ctx.set_state(case[2])
        t, steps = ctx.advance(0, 0.0, t_final, 100000)
        fine = {}
        for f in CONS_2D:
            a = ctx.interior(ctx.get_field(f))[0]
            fine[f] = 0.25 * (a[0::2, 0::2] + a[1::2, 0::2] + a[0::2, 1::2] + a[1::2, 1::2])[None]
        ctx.close()
        return fine, t, steps

    def measure_ensemble(precision, with_clocks=False, with_e2e=False):
        """The batched-ensemble workload in one launch per rank (ranks take
        cost-balanced shares of the tubes); returns this rank's timing and
        per-tube densities (for the mixed-vs-FP64 error)."""
        from semiimplicitfv_b200.shard import rank_share
        inst = ensemble_instances()
        costs = [float(len(c[1].x) - 1) ** 2 for c in inst]
        inst = [inst[k] for k in rank_share(costs, rank, ws)]
        ns = [len(c[1].x) - 1 for c in inst]
        cfg = inst[0][0]
        cfg.precision = precision
        ens = backends.cuda().create_ensemble(cfg, ns, [0.0] * len(ns), [1.0] * len(ns), device=local)
        fids = [f for f in inst[0][2] if f != abi.F_SIGMA]
        packed = {f: torch.from_numpy(ens.pack([c[2][f] for c in inst])).pin_memory() for f in fids}
        for f in fids:
            ens.set_field(f, packed[f].numpy())
        bs = ens.autotune(200)         # also the warm-up launches (long enough that the largest tubes weigh in)
        clk = ClockSampler(local) if with_clocks else None
        if clk:
            clk.__enter__()
        w0 = time.time()
        times, steps, ms = ens.run(ENS_TEND)
        if clk:
            clk.mark(w0, time.time())
            clk.__exit__(None, None, None)
        cu = float(np.dot(np.array(ns, dtype=np.float64), steps))
        rho = [r[ens.ng:-ens.ng].copy() for r in ens.unpack(ens.get_field(abi.F_RHO))]
        out = {"ms": ms, "value": cu / (ms / 1e3), "cell_updates": cu, "block_size": bs, "rho": rho,
               "steps_min": int(steps.min()), "steps_max": int(steps.max()), "ncells": sum(ns),
               "e2e_bytes": len(fids) * ens.ncells * 8, "clocks": clk.summary() if clk else None}
        ens.close()
        if with_e2e:
            # end to end from host buffers: upload the state, run, download it
            ens2 = backends.cuda().create_ensemble(cfg, ns, [0.0] * len(ns), [1.0] * len(ns), device=local)
            t0 = time.perf_counter()
            for f in fids:
                assert ens2.be.fn["ensemble_set_field"](ens2.h, f, ctypes.c_void_p(packed[f].data_ptr()), 0) == 0
            ens2.run(ENS_TEND, block_size=bs)
            for f in fids:
                assert ens2.be.fn["ensemble_get_field"](ens2.h, f, ctypes.c_void_p(packed[f].data_ptr()), 0) == 0
            out["e2e_s"] = time.perf_counter() - t0
            ens2.close()
        return out

    def measure_semi_implicit():
        """Semi-implicit step with IGR and the Jacobi pressure solve: FP64 (the
        reference order, bit-identical to the oracle) and mixed (FP32 inner
        Jacobi sweeps inside FP64 refinement), with the mixed state's L1 / Linf
        error against the FP64 one after the same steps."""
        def run(precision):
            case = cases.acoustic3d(SI_N)
            case[0].precision = precision
            ctx = backends.cuda().create(case[0], case[1], local)
            ctx.set_state(case[2])
            t_sim = 0.0
            for q in range(SI_WARM):                   # step 0 runs the 50-sweep IGR warm start
                t_sim += ctx.step(q, t_sim, -1.0)
            iters = []
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for q in range(SI_STEPS):
                t_sim += ctx.step(SI_WARM + q, t_sim, -1.0)
                iters.append(ctx.last_pressure_iterations())
            torch.cuda.synchronize()
            sec = time.perf_counter() - t0
            fields = {f: ctx.interior(ctx.get_field(f)).copy() for f in (abi.F_RHO, abi.F_RHOU, abi.F_RHOE, abi.F_PRES)}
            fam = ctx.profile_step(SI_WARM + SI_STEPS, t_sim, -1.0)
            ctx.close()
            return case, sec, iters, fields, fam

        case, sec, iters, f64, fam = run(abi.PREC_FP64)
        _, sec_m, iters_m, fmx, fam_m = run(abi.PREC_MIXED)
        cells = SI_N ** 3
        val = cells * SI_STEPS / sec
        val_m = cells * SI_STEPS / sec_m
        kj = float(np.mean(iters))
        nigr = case[0].IGRIters
        bpc = 272 + 32 * nigr + 40 * kj
        err = {}
        for f, name in ((abi.F_RHO, "rho"), (abi.F_RHOU, "rhoU"), (abi.F_RHOE, "rhoE"), (abi.F_PRES, "pres")):
            d = np.abs(fmx[f] - f64[f])
            err[name] = {"l1_rel": float(d.mean() / np.abs(f64[f]).mean()),
                         "linf_rel": float(d.max() / np.abs(f64[f]).max())}
        return {"workload": f"3D acoustic pulse {SI_N}^3 periodic, semi-implicit RK1 + IGR ({nigr} sweeps), "
                            f"WENO5+HLLC, advective CFL 0.8 (dt = maxDt 1e-2), Jacobi tol 1e-6",
                "metric": "cell-updates/s", "value": val, "steps": SI_STEPS, "ms_per_step": sec / SI_STEPS * 1e3,
                "precision": "fp64", "jacobi_iterations": iters,
                "family_ms_per_step": {k: v[0] for k, v in fam.items()},
                "roofline": {"bound": "hbm", "bytes_per_cell_update": bpc, "achieved": bpc * val / 1e9,
                             "unit": "GB/s"},
                "mixed": {"precision": "FP32 inner Jacobi sweeps + FP64 refinement, rest FP64",
                          "value": val_m, "ms_per_step": sec_m / SI_STEPS * 1e3, "jacobi_iterations": iters_m,
                          "family_ms_per_step": {k: v[0] for k, v in fam_m.items()},
                          "error_vs_fp64": err}}

    def measure_semi_2d_periodic():
        """Semi-implicit steps on a periodic 2D mesh with IGR and the
        Gauss-Seidel pressure solve (the reference's 2D semi-implicit examples
        use GaussSeidelPressureSolver): both run as the persistent 2D
        wavefront (k_march_gs); the same steps with the tiled sweeps
        (SIFV_GS_MARCH=0) beside them.  Device time per step from CUDA events
        around whole steps after the warm-start step; results are bit-identical
        between the two."""
        out = {}
        prev = os.environ.get("SIFV_GS_MARCH")
        try:
            for name, mode in (("wavefront", None), ("tiles", "0")):
                if mode is None:
                    os.environ.pop("SIFV_GS_MARCH", None)
                else:
                    os.environ["SIFV_GS_MARCH"] = mode
                case = cases.acoustic_box(SI2_N, SI2_N)
                ctx = backends.cuda().create(case[0], case[1], local)
                ctx.set_state(case[2])
                ctx.set_pressure_solver(abi.PRESSURE_GAUSS_SEIDEL)
                t_sim = 0.0
                for q in range(2):                     # step 0: the 20-sweep IGR warm start
                    t_sim += ctx.step(q, t_sim, -1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                iters = []
                torch.cuda.synchronize()
                e0.record()
                for q in range(SI2_STEPS):
                    t_sim += ctx.step(2 + q, t_sim, -1.0)
                    iters.append(ctx.last_pressure_iterations())
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / SI2_STEPS
                fam = ctx.profile_step(2 + SI2_STEPS, t_sim, -1.0)
                out[name] = {"ms_per_step": ms, "value": SI2_N * SI2_N / (ms * 1e-3),
                             "gauss_seidel_iterations": iters,
                             "family_ms_per_step": {k: v[0] for k, v in fam.items()}}
                ctx.close()
        except Exception as e:   # a failed extra measurement must not cost the bench line
            out["error"] = str(e)[:200]
        finally:
            if prev is None:
                os.environ.pop("SIFV_GS_MARCH", None)
            else:
                os.environ["SIFV_GS_MARCH"] = prev
        out["workload"] = (f"2D acoustic pulse {SI2_N}^2, all faces periodic, semi-implicit RK1 + IGR (5 sweeps), "
                           f"Gauss-Seidel pressure solve (tol 1e-8, at most 300 iterations), WENO5+HLLC")
        out["metric"] = "cell-updates/s"
        return out

    def measure_pressure_solvers():
        """Device time of the pressure solve of the first step after the
        warm-up of the 256^3 semi-implicit workload with each pressure solver
        (reference-ordered Jacobi and Gauss-Seidel, and PCG with a multigrid
        V-cycle in place of Hypre's PCG + PFMG), from the per-family CUDA
        events of sifv_profile_step, with the iteration count."""
        out = {}
        for name, kind in (("jacobi", abi.PRESSURE_JACOBI), ("gauss_seidel", abi.PRESSURE_GAUSS_SEIDEL),
                           ("pcg_mg", abi.PRESSURE_PCG_MG)):
            try:
                case = cases.acoustic3d(SI_N)
                ctx = backends.cuda().create(case[0], case[1], local)
                ctx.set_state(case[2])
                ctx.set_pressure_solver(kind)
                t_sim = 0.0
                for q in range(SI_WARM):
                    t_sim += ctx.step(q, t_sim, -1.0)
                fam = ctx.profile_step(SI_WARM, t_sim, -1.0)
                out[name] = {"ms": fam[name][0], "iterations": ctx.last_pressure_iterations(),
                             "step_ms": sum(v[0] for v in fam.values())}
                ctx.close()
            except Exception as e:   # a failed extra measurement must not cost the bench line
                out[name] = {"error": str(e)[:200]}
        return out

    def measure_adjoint():
        """Forward (recording) and reverse sweep of the vortex adjoint."""
        case = cases.vortex2d(ADJ_N)
        ctx = backends.cuda().create(case[0], case[1], local)
        ctx.set_state(case[2])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, steps = ctx.adjoint_forward(0, 0.0, ADJ_TEND, 0, ADJ_EVERY)
        fwd_s = time.perf_counter() - t0
        fids = [abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE]
        # J = sum over cells with r < 1 of p^2 dA at t_end: dJ/dU = 2 p dA dp/dU,
        # p = (gamma - 1) (E - (m_x^2 + m_y^2) / (2 rho))
        U = [ctx.get_field(f) for f in fids]
        g1 = case[0].gamma - 1.0
        rho, mx, my, E = U
        with np.errstate(divide="ignore", invalid="ignore"):
            p = g1 * (E - 0.5 * (mx * mx + my * my) / rho)
            u, v = mx / rho, my / rho
        x = case[1].x
        xc = 0.5 * (x[:-1] + x[1:])
        X, Y = np.meshgrid(xc, xc, indexing="xy")
        dA = (x[1] - x[0]) ** 2
        disk = np.zeros(ctx.shape, dtype=bool)
        ctx.interior(disk)[...] = (X * X + Y * Y < 1.0)[None]
        w = np.where(disk, 2.0 * p * dA, 0.0)
        seeds = {abi.F_RHO: w * g1 * 0.5 * (u * u + v * v), abi.F_RHOU: -w * g1 * u, abi.F_RHOV: -w * g1 * v,
                 abi.F_RHOE: w * g1}
        seeds = {f: np.where(disk, a, 0.0) for f, a in seeds.items()}
        for f in fids:
            ctx.adjoint_set_seed(f, seeds[f])
        ctx.adjoint_backward()                       # warm-up (allocates the stage store)
        for f in fids:
            ctx.adjoint_set_seed(f, seeds[f])
        bwd_ms = ctx.adjoint_backward()
        g64 = {f: ctx.interior(ctx.adjoint_get_gradient(f)).copy() for f in fids}
        # the same reverse sweep with FP32 local Jacobians
        ctx.adjoint_set_precision(abi.PREC_MIXED)
        for f in fids:
            ctx.adjoint_set_seed(f, seeds[f])
        ctx.adjoint_backward()
        for f in fids:
            ctx.adjoint_set_seed(f, seeds[f])
        bwd32_ms = ctx.adjoint_backward()
        err32 = {}
        for f, name in zip(fids, ("rho", "rhoU", "rhoV", "rhoE")):
            d = np.abs(ctx.interior(ctx.adjoint_get_gradient(f)) - g64[f])
            err32[name] = {"l1_rel": float(d.mean() / np.abs(g64[f]).mean()),
                           "linf_rel": float(d.max() / np.abs(g64[f]).max())}
        cells = ADJ_N * ADJ_N
        ctx.close()
        val = cells * steps / (bwd_ms / 1e3)
        return {"workload": f"isentropic vortex {ADJ_N}x{ADJ_N} periodic, WENO5+HLLC SSP-RK3 CFL0.6 to t={ADJ_TEND}, "
                            f"gradient of J = sum_(r<1) p^2 dA at t_end w.r.t. U(0), checkpoint every {ADJ_EVERY} "
                            f"steps",
                "metric": "adjoint cell-updates/s", "value": val, "steps": steps,
                "backward_seconds": bwd_ms / 1e3, "forward_seconds_recording": fwd_s,
                "forward_value": cells * steps / fwd_s, "precision": "fp64",
                "fp32": {"precision": "FP32 local Jacobians in the reverse sweep (forward, adjoint state and "
                                      "share accumulation FP64)",
                         "value": cells * steps / (bwd32_ms / 1e3), "backward_seconds": bwd32_ms / 1e3,
                         "error_vs_fp64_gradient": err32},
                "roofline": {"bound": "hbm", "bytes_per_cell_update": ADJ_BYTES_PER_CELL_UPDATE,
                             "achieved": ADJ_BYTES_PER_CELL_UPDATE * val / 1e9, "unit": "GB/s"}}

    if args.profile_case:
        # a small instance of one of the other workloads (for ncu captures)
        t0 = time.perf_counter()
        if args.profile_case == "semi":
            case = cases.acoustic3d(args.n)
            ctx = backends.cuda().create(case[0], case[1], local)
            ctx.set_state(case[2])
            t_sim = 0.0
            for q in range(args.steps):
                t_sim += ctx.step(q, t_sim, -1.0)
            ctx.close()
        elif args.profile_case == "adjoint":
            case = cases.vortex2d(args.n)
            ctx = backends.cuda().create(case[0], case[1], local)
            ctx.set_state(case[2])
            ctx.adjoint_forward(0, 0.0, 10.0, args.steps, ADJ_EVERY)
            seed = np.zeros(ctx.shape)
            ctx.interior(seed)[...] = 1.0
            for f in (abi.F_RHO, abi.F_RHOU, abi.F_RHOV, abi.F_RHOE):
                ctx.adjoint_set_seed(f, seed)
            ctx.adjoint_backward()
            ctx.close()
        else:
            inst = ensemble_instances(count=args.n, nmin=256, nmax=2048)
            ns = [len(c[1].x) - 1 for c in inst]
            cfg = inst[0][0]
            cfg.precision = args.precision if args.precision in (0, 1) else abi.PREC_MIXED
            ens = backends.cuda().create_ensemble(cfg, ns, [0.0] * len(ns), [1.0] * len(ns), device=local)
            for f in inst[0][2]:
                if f != abi.F_SIGMA:
                    ens.set_field(f, ens.pack([c[2][f] for c in inst]))
            ens.run(ENS_TEND, max_steps=args.steps, block_size=512)
            ens.close()
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_case": args.profile_case, "n": args.n, "steps": args.steps,
                              "seconds": time.perf_counter() - t0}), flush=True)
        return

    if args.kernels_only:
        r = measure(args.precision)
        if rank == 0:
            print(json.dumps({"kernels_only": True, "n": n, "precision": PREC_NAMES[args.precision],
                              "ms_per_step": r["ms"] / args.steps, "value": r["value"],
                              "units_per_warp": r["tuned"]}), flush=True)
        if ws > 1:
            torch.distributed.destroy_process_group()
        return

    main = measure(args.precision, with_clocks=True, with_e2e=True)
    extra = {}
    for p in (0, 1, 2):
        if p != args.precision and not args.quick:
            extra[PREC_NAMES[p]] = measure(p)
    adj = None
    if ws == 1 and not args.quick and not args.no_adjoint:
        adj = measure_adjoint()
    semi = None
    if ws == 1 and not args.quick and not args.no_semi:
        semi = measure_semi_implicit()
    ens = None
    if not args.quick and not args.no_ensemble:
        from semiimplicitfv_b200.shard import max_over_ranks as mor, sum_over_ranks as sor
        barrier()
        emx = measure_ensemble(abi.PREC_MIXED, with_clocks=(rank == 0), with_e2e=True)
        barrier()
        e64 = measure_ensemble(abi.PREC_FP64)
        rel = [np.abs(a - b).mean() / np.abs(b).mean() for a, b in zip(emx["rho"], e64["rho"])]
        linf = [np.abs(a - b).max() / np.abs(b).max() for a, b in zip(emx["rho"], e64["rho"])]
        dev = "cuda" if ws > 1 else None
        for e in (emx, e64):     # whole job: all tubes over the slowest rank's time
            e["ms"] = mor(e["ms"], dev)
            e["cell_updates"] = sor(e["cell_updates"], dev)
            e["ncells"] = int(sor(e["ncells"], dev))
            e["value"] = e["cell_updates"] / (e["ms"] / 1e3)
            e["steps_min"] = -int(mor(-e["steps_min"], dev))
            e["steps_max"] = int(mor(e["steps_max"], dev))
        emx["e2e"] = emx["cell_updates"] / mor(emx["e2e_s"], dev)
        ens = {"mixed": emx, "fp64": e64, "l1_rel_max": mor(float(max(rel)), dev),
               "l1_rel_mean": float(np.mean(rel)), "linf_rel_max": mor(float(max(linf)), dev)}
    accuracy = None
    if ws == 1 and not args.quick and PREC_NAMES[0] in extra:
        # every result's L1 / L-inf error against the FP64 (reference-ordered)
        # state after the same steps, and against the 2n x 2n FP64 solution
        # at the same time (the discretisation error)
        runs = {PREC_NAMES[args.precision]: main, **extra}
        ref = runs[PREC_NAMES[0]]
        fine, t_fine, fine_steps = measure_fine(ref["t"])

        def err(a, b):
            d = np.abs(a - b)
            return {"l1": float(d.mean()), "l1_rel": float(d.mean() / np.abs(b).mean()),
                    "linf_rel": float(d.max() / np.abs(b).max())}
        accuracy = {"vs_fp64": {}, "vs_fine_grid": {},
                    "fine_grid": f"{2 * n}x{2 * n} reference-ordered FP64 to the same t = {t_fine:.6e} "
                                 f"({fine_steps} steps), 2x2-block averages"}
        for name, r in runs.items():
            if name != PREC_NAMES[0]:
                accuracy["vs_fp64"][name] = {v: err(r["state"][f], ref["state"][f]) for f, v in zip(CONS_2D, CONS_NAMES_2D)}
            accuracy["vs_fine_grid"][name] = {v: err(r["state"][f], fine[f]) for f, v in zip(CONS_2D, CONS_NAMES_2D)}
        d64 = accuracy["vs_fine_grid"][PREC_NAMES[0]]
        for name in runs:
            if name != PREC_NAMES[0]:
                accuracy["vs_fine_grid"][name]["l1_over_fp64"] = max(
                    accuracy["vs_fine_grid"][name][v]["l1"] / max(d64[v]["l1"], 1e-300) for v in CONS_NAMES_2D)
        for r in runs.values():
            r.pop("state", None)
    ms = main["ms"]
    value = main["value"]
    launches = main["launches"]
    e2e_value = main["e2e"]

    class _Clk:
        def summary(self):
            return main["clocks"]
    clk = _Clk()

    peak, peak_kind = _peaks()
    step_achieved = BYTES_PER_CELL_UPDATE * cells * args.steps / (ms / 1e3) / 1e9
    fam = main["families"]
    dom = max(fam, key=lambda k: fam[k][0])
    dom_ms = fam[dom][0] / fam[dom][1]
    dom_bytes = KERNEL_BYTES_PER_CELL_2D.get(dom, float("nan")) * cells
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    cap = NCU_CAPTURE.get((args.precision, dom))
    sha = _kernel_sources_sha()
    fresh = cap is not None and cap.get("sha") == sha
    traffic = cap["dram_bytes_per_cell"] * cells if fresh else None
    fp64_peak = None
    try:
        tf = ctypes.c_double()
        if backends.cuda().lib.sifv_fp64_peak_probe(5, ctypes.byref(tf)) == 0:
            fp64_peak = tf.value
    except Exception:
        pass
    result = None
    if rank == 0:
        kind = "reference" if backends.reference(release=True) is not None else "port"
        if kind == "reference":   # bounded sample: 1 + 2 steps of the same grid on all host cores
            cpu_cores = _host_cores()
            cpu, cpu_sec, cpu_dims = reference_decomposed_rate(n, 1, 2, cpu_cores)
            cpu_sample = (f"{n}x{n}, 1 warm-up + 2 timed steps of the full grid, decomposed over {cpu_cores} MPI "
                          f"ranks ({cpu_dims[0]}x{cpu_dims[1]}, threads through the MPI shim), Release flags")
        else:
            cpu_cores, cpu = 1, cpu_rate(kind, 768, 3)
            cpu_sample = "C restatement on one core, 768x768 instance, 3 steps"
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if args.precision != 1 else "f32-bulk/f64-state",
            "data": "synthetic",
            "precision": PREC_NAMES[args.precision],
            "parallelism": (f"slab decomposition over {ws} GPUs (rows split along y, 3-row halo exchange per RK "
                            f"stage and dt all-reduce over NCCL)" if ws > 1 else "1 GPU"),
            "config": workload_config(n),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": (f"ncu dram bytes per cell of one {dom} launch (average over the 3 "
                                            f"stage launches of a step, 2048^2 case) x {cells} cells" if fresh else
                                            f"no ncu capture of the current {dom} sources ({sha})"),
                         "kernel": dom, "bytes_per_launch": dom_bytes, "ms_per_launch": dom_ms,
                         "peak_source": peak_kind,
                         "step": {"achieved": step_achieved, "frac": step_achieved / peak,
                                  "bytes_per_cell_update": BYTES_PER_CELL_UPDATE},
                         "kernel_ms_per_step": {k: v[0] / 2 for k, v in fam.items()},
                         "compute_co_bound": {
                             "fp64_peak_tflops": fp64_peak,
                             "fp64_peak_source": "measured: FP64 FMA throughput probe (sifv_fp64_peak_probe)",
                             "fp64_inst_per_cell": cap.get("fp64_inst_per_cell") if fresh else None,
                             "fp64_inst_rate_frac": (cap["fp64_inst_per_cell"] * cells / (dom_ms / 1e3) /
                                                     (fp64_peak * 1e12 / 2.0)
                                                     if fresh and fp64_peak and cap.get("fp64_inst_per_cell")
                                                     else None),
                             "note": "FP64 instructions per cell from the ncu capture over the probe's FMA "
                                     "instruction rate"}},
            "cpu_baseline": {"value": cpu, "unit": UNIT, "cores": cpu_cores, "kind": kind, "sample": cpu_sample},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": main["e2e_bytes"],
                    "d2h_bytes_per_step": main["e2e_bytes"] + 8,
                    "api": "per step: sifv_set_field x7 from pinned host buffers, sifv_step (dt to the host), "
                           "sifv_get_field x7 (host-authoritative drop-in)",
                    "resident_value": main["e2e_resident"],
                    "resident_api": "sifv_step only, state resident on the GPU (dt to the host each step)"},
            "gpu_launches": launches,
            "autotune": {"units_per_warp": main["tuned"],
                         "what": "work units (30-column strip x row segment) per resident warp of the fused "
                                 "stage kernel, chosen by timing 1-4 (sifv_autotune)"},
            "clocks": clk.summary(),
            "other_precisions": {k: {"value": v["value"], "ms_per_step": v["ms"] / args.steps,
                                     "roofline_frac": BYTES_PER_CELL_UPDATE * v["value"] / 1e9 / peak,
                                     "error_vs_fp64": (accuracy or {}).get("vs_fp64", {}).get(k)}
                                 for k, v in extra.items()},
            "error_vs_fp64": (accuracy or {}).get("vs_fp64", {}).get(PREC_NAMES[args.precision]),
            "accuracy": accuracy,
        }
        if semi is not None:
            semi["roofline"]["peak"] = peak
            semi["roofline"]["frac"] = semi["roofline"]["achieved"] / peak
            srate, ssample = semi_cpu_rate(kind)
            semi["cpu_baseline"] = {"value": srate, "unit": UNIT, "cores": 1, "kind": kind, "sample": ssample}
            semi["pressure_solvers"] = measure_pressure_solvers()
            result["semi_implicit"] = semi
            result["semi_implicit_2d_periodic"] = measure_semi_2d_periodic()
        if adj is not None:
            adj["roofline"]["peak"] = peak
            adj["roofline"]["frac"] = adj["roofline"]["achieved"] / peak
            result["adjoint"] = adj
        if ens is not None:
            mx, f64 = ens["mixed"], ens["fp64"]
            ens_cpu, ens_sample = ensemble_cpu_rate(kind, os.cpu_count() or 1)
            result["ensemble"] = {
                "workload": f"{ENS_COUNT} two-phase water-air tubes, cells log-uniform [{ENS_NMIN},{ENS_NMAX}] "
                            f"(seed {ENS_SEED}, {mx['ncells']} cells), WENO5 + mixture HLLC, SSP-RK3 CFL0.5, "
                            f"t_end={ENS_TEND}, one launch per GPU",
                "scaling": "strong (the tubes are divided across GPUs by cost, cells^2)",
                "metric": "cell-updates/s", "value": mx["value"], "precision": "mixed-fp32-bulk",
                "seconds": mx["ms"] / 1e3, "cell_updates": mx["cell_updates"],
                "steps_min_max": [mx["steps_min"], mx["steps_max"]], "threads_per_tube": mx["block_size"],
                "fp64": {"value": f64["value"], "seconds": f64["ms"] / 1e3, "threads_per_tube": f64["block_size"]},
                "mixed_vs_fp64_rho": {"l1_rel_max": ens["l1_rel_max"], "l1_rel_mean": ens["l1_rel_mean"],
                                      "linf_rel_max": ens["linf_rel_max"]},
                "roofline": {"bound": "hbm", "bytes_per_cell_update": ENS_BYTES_PER_CELL_UPDATE,
                             "achieved": ENS_BYTES_PER_CELL_UPDATE * mx["value"] / 1e9, "peak": peak,
                             "unit": "GB/s", "frac": ENS_BYTES_PER_CELL_UPDATE * mx["value"] / 1e9 / peak},
                "e2e": {"value": mx["e2e"], "h2d_bytes": mx["e2e_bytes"], "d2h_bytes": mx["e2e_bytes"],
                        "api": "sifv_ensemble_set_field x9, sifv_ensemble_run, sifv_ensemble_get_field x9"},
                "cpu_baseline": {"value": ens_cpu, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": kind,
                                 "sample": ens_sample},
                "clocks": mx["clocks"],
            }
        print(json.dumps(result), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--precision", type=int, default=2, choices=[0, 1, 2],
                    help="0 reference-ordered FP64, 1 mixed (FP32 bulk), 2 fast FP64 (default)")
    ap.add_argument("--quick", action="store_true", help="skip the other precisions and the ensemble")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble workload")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint workload")
    ap.add_argument("--no-semi", action="store_true", help="skip the semi-implicit 3D workload")
    ap.add_argument("--profile-case", choices=["semi", "adjoint", "ensemble"], default=None,
                    help="run a small instance of another workload (--n: cells per axis, or tubes) and exit")
    ap.add_argument("--units-per-warp", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="fix the work units per warp of the 2D fused stage (0: choose by sifv_autotune)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the device-timed step loop (no clocks, e2e, CPU baseline): a small case to profile")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
