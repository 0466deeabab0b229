"""ctypes mirror of the C ABI in ``include/sifv.h``.

The same structs and call shapes serve every library that implements the
ABI: the CUDA library of this package (symbol prefix ``sifv_``) and, in the
tests only, the CPU oracles (``sifvo_`` for the C restatement, ``sifvr_``
for the reference build).  ``Config`` mirrors ``SimulationConfig``
(include/SimulationConfig.hpp:72-210 of SemiImplicitFV) field for field and
``config_defaults`` reproduces its member initialisers.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

MAX_PHASES = 8

# status codes
OK, NOT_CONVERGED = 0, 1
ERR_BAD_CONFIG, ERR_BAD_ARG, ERR_CUDA, ERR_NAN = -1, -2, -3, -4
ERR_UNSUPPORTED, ERR_TIMEOUT, ERR_NO_DEVICE = -5, -6, -7

# ReconstructionOrder (include/SimulationConfig.hpp:13-20)
WENO1, WENO3, WENO5, UPWIND1, UPWIND3, UPWIND5 = range(6)
# RiemannSolverType (include/RiemannSolver.hpp:16)
LF, RUSANOV, HLLC = range(3)
# BoundaryCondition (include/RectilinearMesh.hpp:14-20)
BC_SYMMETRY, BC_OUTFLOW, BC_PERIODIC, BC_SLIPWALL, BC_NOSLIPWALL = range(5)
BC_EXCHANGE = 16   # a face shared with a neighbouring rank (ghost layers filled by the halo exchange)
EOS_IDEAL, EOS_STIFFENED = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP64_FAST = 0, 1, 2

# field identifiers (SolutionState members, include/SolutionState.hpp:73-113)
F_RHO, F_RHOU, F_RHOV, F_RHOW, F_RHOE = 0, 1, 2, 3, 4
F_VELU, F_VELV, F_VELW, F_PRES, F_SIGMA = 5, 6, 7, 8, 9


def F_ALPHARHO(ph: int) -> int:
    return 16 + ph


def F_ALPHA(ph: int) -> int:
    return 32 + ph


class Config(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nGhost", C.c_int), ("RKOrder", C.c_int),
        ("useIGR", C.c_int), ("semiImplicit", C.c_int), ("reconOrder", C.c_int),
        ("wenoEps", C.c_double),
        ("riemannSolver", C.c_int), ("eosKind", C.c_int),
        ("gamma", C.c_double), ("pInf", C.c_double),
        ("cfl", C.c_double), ("constDt", C.c_double), ("maxDt", C.c_double), ("minDt", C.c_double),
        ("siCfl", C.c_double), ("siMaxDt", C.c_double), ("siMinDt", C.c_double),
        ("maxPressureIters", C.c_int), ("pressureTol", C.c_double),
        ("alphaCoeff", C.c_double), ("IGRIters", C.c_int), ("IGRWarmStartIters", C.c_int),
        ("nPhases", C.c_int),
        ("phaseGamma", C.c_double * MAX_PHASES), ("phasePInf", C.c_double * MAX_PHASES),
        ("alphaMin", C.c_double),
        ("bfA", C.c_double * 3), ("bfB", C.c_double * 3), ("bfC", C.c_double * 3), ("bfD", C.c_double * 3),
        ("precision", C.c_int),
        ("mu", C.c_double), ("phaseMu", C.c_double * MAX_PHASES), ("nPhaseMu", C.c_int),
        ("stSigma", C.c_double), ("stEpsGradAlpha", C.c_double),
    ]


class Mesh(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xNodes", C.POINTER(C.c_double)), ("yNodes", C.POINTER(C.c_double)),
        ("zNodes", C.POINTER(C.c_double)),
        ("bc", C.c_int * 6),
    ]


def config_defaults(**overrides) -> Config:
    """SimulationConfig defaults (include/SimulationConfig.hpp:22-92), IdealGasEOS(1.4)."""
    c = Config()
    c.dim, c.nGhost, c.RKOrder = 3, 2, 1
    c.useIGR, c.semiImplicit = 0, 0
    c.reconOrder, c.wenoEps = WENO1, 1e-6
    c.riemannSolver, c.eosKind, c.gamma, c.pInf = HLLC, EOS_IDEAL, 1.4, 0.0
    c.cfl, c.constDt, c.maxDt, c.minDt = 0.8, -1.0, 1e-2, 1e-12
    c.siCfl, c.siMaxDt, c.siMinDt = 0.8, 1e-2, 1e-12
    c.maxPressureIters, c.pressureTol = 100, 1e-8
    c.alphaCoeff, c.IGRIters, c.IGRWarmStartIters = 1.0, 5, 50
    c.nPhases, c.alphaMin = 0, 1e-8
    c.precision = PREC_FP64
    c.mu, c.nPhaseMu = 0.0, 0
    c.stSigma, c.stEpsGradAlpha = 0.0, 1e-8
    for k, v in overrides.items():
        if k in ("phaseGamma", "phasePInf"):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = x
        elif k in ("bfA", "bfB", "bfC", "bfD"):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            if not hasattr(c, k):
                raise AttributeError(f"unknown config field {k}")
            setattr(c, k, v)
    return c


def linspace_nodes(n: int, lo: float, hi: float) -> np.ndarray:
    """Global node array of Runtime::createUniformMesh: a + (b - a) * i / (n - 1)
    with n = cells + 1 points (src/Runtime.cpp:12-17), evaluated in the same order."""
    npts = n + 1
    i = np.arange(npts, dtype=np.float64)
    return lo + ((hi - lo) * i) / float(npts - 1)


class MeshSpec:
    """Node arrays + boundary conditions; keeps the numpy buffers alive."""

    def __init__(self, x: np.ndarray, y: Optional[np.ndarray] = None, z: Optional[np.ndarray] = None,
                 bc: Sequence[int] = (BC_OUTFLOW,) * 6):
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
        self.z = None if z is None else np.ascontiguousarray(z, dtype=np.float64)
        self.bc = list(bc)

    def cstruct(self) -> Mesh:
        m = Mesh()
        dp = C.POINTER(C.c_double)
        m.nx = len(self.x) - 1
        m.ny = 1 if self.y is None else len(self.y) - 1
        m.nz = 1 if self.z is None else len(self.z) - 1
        m.xNodes = self.x.ctypes.data_as(dp)
        m.yNodes = self.y.ctypes.data_as(dp) if self.y is not None else dp()
        m.zNodes = self.z.ctypes.data_as(dp) if self.z is not None else dp()
        for f in range(6):
            m.bc[f] = self.bc[f]
        return m


PRESSURE_JACOBI, PRESSURE_GAUSS_SEIDEL, PRESSURE_PCG_MG = 0, 1, 2
IB_CIRCLE, IB_RECTANGLE, IB_CYLINDER, IB_PRISM = 0, 1, 2, 3
IB_NOSLIP, IB_SLIP = 0, 1
CELL_FLUID, CELL_GHOST, CELL_DEAD = 0, 1, 2


class IbBody(C.Structure):
    _fields_ = [("shape", C.c_int), ("wall", C.c_int), ("axis", C.c_int), ("p", C.c_double * 6)]


def ib_body(shape: int, params, wall: int = IB_NOSLIP, axis: int = 2) -> IbBody:
    b = IbBody()
    b.shape, b.wall, b.axis = shape, wall, axis
    for i, v in enumerate(params):
        b.p[i] = v
    return b


class VtkFields(C.Structure):
    _fields_ = [("pres", C.c_void_p), ("sigma", C.c_void_p), ("rhoE", C.c_void_p), ("vel", C.c_void_p * 3),
                ("mom", C.c_void_p * 3), ("rho", C.c_void_p), ("alphaRho", C.c_void_p * MAX_PHASES),
                ("alpha", C.c_void_p * MAX_PHASES)]


class TimeLoop(C.Structure):
    _fields_ = [("endTime", C.c_double), ("outputInterval", C.c_double), ("printInterval", C.c_int),
                ("checkNaN", C.c_int), ("step0", C.c_int), ("batch", C.c_int)]


class LoopResult(C.Structure):
    _fields_ = [("time", C.c_double), ("steps", C.c_int), ("outputs", C.c_int), ("nanField", C.c_int),
                ("nanCell", C.c_longlong), ("nanTime", C.c_double), ("nanStep", C.c_int)]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_double, C.c_double)
# sifv_comm_t: halo exchange and dt reduction of a decomposed run
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_void_p)
ALLREDUCE_MIN_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)


class Comm(C.Structure):
    _fields_ = [("exchange", EXCHANGE_FN), ("allreduce_min", ALLREDUCE_MIN_FN), ("user", C.c_void_p),
                ("allreduce_max", ALLREDUCE_MIN_FN)]


class AbiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"status {status}: {msg}")
        self.status = status


_SIGS = {
    "create": (C.c_int, [C.POINTER(Config), C.POINTER(Mesh), C.c_int, C.POINTER(C.c_void_p)]),
    "destroy": (C.c_int, [C.c_void_p]),
    "last_error": (C.c_char_p, [C.c_void_p]),
    "extents": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "total_cells": (C.c_size_t, [C.c_void_p]),
    "set_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "get_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "last_pressure_iterations": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "pressure_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "igr_solve": (C.c_int, [C.c_void_p, C.c_int]),
    "acoustic_dt": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "advective_dt": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "convert_cons_to_prim": (C.c_int, [C.c_void_p]),
    "apply_bc": (C.c_int, [C.c_void_p]),
}

_OPTIONAL_SIGS = {
    "advance": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                          C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "synchronize": (C.c_int, [C.c_void_p]),
    "set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "field_device_ptr": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "last_step_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "set_pressure_solver": (C.c_int, [C.c_void_p, C.c_int]),
    "config_validate": (C.c_int, [C.POINTER(Config)]),
    "profile_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_char_p, C.c_int,
                               C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
    "adjoint_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                  C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "adjoint_schedule": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int)]),
    "adjoint_set_seed": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "adjoint_backward": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "adjoint_get_gradient": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "tangent_set_direction": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "tangent_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                                  C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "tangent_get": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "adjoint_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "ensemble_create": (C.c_int, [C.POINTER(Config), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_void_p)]),
    "ensemble_destroy": (C.c_int, [C.c_void_p]),
    "ensemble_last_error": (C.c_char_p, [C.c_void_p]),
    "ensemble_layout": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "ensemble_set_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "ensemble_get_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "ensemble_run": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_double),
                               C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "ensemble_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "check_nan": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "set_immersed_bodies": (C.c_int, [C.c_void_p, C.POINTER(IbBody), C.c_int]),
    "ib_cell_types": (C.c_int, [C.c_void_p, C.c_void_p]),
    "apply_ib_ghost_cells": (C.c_int, [C.c_void_p]),
    "vtk_open": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Config), C.POINTER(Mesh), C.c_int,
                           C.POINTER(C.c_void_p)]),
    "vtk_write_host": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(VtkFields)]),
    "vtk_write": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "vtk_flush": (C.c_int, [C.c_void_p]),
    "vtk_close": (C.c_int, [C.c_void_p]),
    "vtk_last_error": (C.c_char_p, [C.c_void_p]),
    "run_time_loop": (C.c_int, [C.c_void_p, C.POINTER(TimeLoop), C.c_void_p, PROGRESS_FN, C.c_void_p,
                                C.POINTER(LoopResult)]),
    "reference_time_loop": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double, C.c_double, C.c_int,
                                      C.POINTER(C.c_int)]),
    "set_comm": (C.c_int, [C.c_void_p, C.POINTER(Comm)]),
    "autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "set_work_units": (C.c_int, [C.c_void_p, C.c_int]),
}


class Backend:
    """A loaded library implementing the ABI under ``prefix``."""

    def __init__(self, lib: C.CDLL, prefix: str, name: str = ""):
        self.lib = lib
        self.prefix = prefix
        self.name = name or prefix
        self.fn = {}
        for k, (res, args) in _SIGS.items():
            f = getattr(lib, prefix + k)
            f.restype, f.argtypes = res, args
            self.fn[k] = f
        for k, (res, args) in _OPTIONAL_SIGS.items():
            f = getattr(lib, prefix + k, None)
            if f is not None:
                f.restype, f.argtypes = res, args
                self.fn[k] = f

    def error(self, ctx=None) -> str:
        m = self.fn["last_error"](ctx)
        return m.decode() if m else ""

    def create(self, cfg: Config, mesh: MeshSpec, device: int = 0) -> "Context":
        h = C.c_void_p()
        ms = mesh.cstruct()
        st = self.fn["create"](C.byref(cfg), C.byref(ms), device, C.byref(h))
        if st != OK:
            raise AbiError(st, self.error(None))
        return Context(self, h, cfg, mesh)

    def create_ensemble(self, cfg: Config, n_cells: Sequence[int], x_lo: Sequence[float],
                        x_hi: Sequence[float], bc=(BC_OUTFLOW, BC_OUTFLOW), device: int = 0) -> "Ensemble":
        if "ensemble_create" not in self.fn:
            raise AbiError(ERR_UNSUPPORTED, f"{self.name} has no ensemble entry points")
        k = len(n_cells)
        nc = (C.c_int * k)(*[int(v) for v in n_cells])
        lo = (C.c_double * k)(*[float(v) for v in x_lo])
        hi = (C.c_double * k)(*[float(v) for v in x_hi])
        b = (C.c_int * 2)(int(bc[0]), int(bc[1]))
        h = C.c_void_p()
        st = self.fn["ensemble_create"](C.byref(cfg), k, nc, lo, hi, b, device, C.byref(h))
        if st != OK:
            raise AbiError(st, self.fn["ensemble_last_error"](None).decode())
        return Ensemble(self, h, cfg, list(n_cells))


class VtkSession:
    """VTKSession-compatible output (.pvd / .pvtr / .vtr) of one rank."""

    def __init__(self, be: "Backend", directory: str, base: str, cfg: Config, mesh: MeshSpec, threads: int = 0):
        if "vtk_open" not in be.fn:
            raise AbiError(ERR_UNSUPPORTED, f"{be.name} has no VTK entry points")
        self.be = be
        self.h = C.c_void_p()
        ms = mesh.cstruct()
        st = be.fn["vtk_open"](directory.encode(), base.encode(), C.byref(cfg), C.byref(ms), threads, C.byref(self.h))
        if st != OK:
            raise AbiError(st, be.fn["vtk_last_error"](None).decode())

    def _check(self, st: int):
        if st != OK:
            raise AbiError(st, self.be.fn["vtk_last_error"](self.h).decode())

    def write_host(self, time: float, fields: dict):
        """fields: SIFV_F_* id -> full (ghosted) float64 array."""
        keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in fields.items()}
        f = VtkFields()
        ptr = lambda fid: keep[fid].ctypes.data if fid in keep else None
        f.pres, f.sigma, f.rhoE, f.rho = ptr(F_PRES), ptr(F_SIGMA), ptr(F_RHOE), ptr(F_RHO)
        for d, (v, m) in enumerate(((F_VELU, F_RHOU), (F_VELV, F_RHOV), (F_VELW, F_RHOW))):
            f.vel[d], f.mom[d] = ptr(v), ptr(m)
        for p in range(MAX_PHASES):
            f.alphaRho[p], f.alpha[p] = ptr(F_ALPHARHO(p)), ptr(F_ALPHA(p))
        self._check(self.be.fn["vtk_write_host"](self.h, time, C.byref(f)))

    def write(self, ctx: "Context", time: float):
        st = self.be.fn["vtk_write"](self.h, ctx.h, time)
        if st != OK:
            raise AbiError(st, self.be.error(ctx.h))

    def flush(self):
        self._check(self.be.fn["vtk_flush"](self.h))

    def close(self):
        if self.h:
            h, self.h = self.h, None
            st = self.be.fn["vtk_close"](h)
            if st != OK:
                raise AbiError(st, "VTK write failed")

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """Independent 1D problems of different sizes advanced together
    (sifv_ensemble_*).  Fields are packed instance after instance with
    ghosts; ``offsets[k]:offsets[k + 1]`` is instance k's slice."""

    def __init__(self, be: "Backend", handle: C.c_void_p, cfg: Config, n_cells):
        self.be, self.h, self.cfg, self.n_cells = be, handle, cfg, n_cells
        k = len(n_cells)
        off = (C.c_longlong * (k + 1))()
        self._check(be.fn["ensemble_layout"](handle, off))
        self.offsets = np.array(off[:], dtype=np.int64)
        self.ncells = int(self.offsets[-1])
        self.ng = cfg.nGhost

    def _check(self, st: int) -> int:
        if st < 0:
            raise AbiError(st, self.be.fn["ensemble_last_error"](self.h).decode())
        return st

    def close(self):
        if self.h:
            self.be.fn["ensemble_destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack(self, per_instance) -> np.ndarray:
        """Concatenate per-instance arrays (each n + 2 nGhost long)."""
        out = np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1) for a in per_instance])
        assert out.size == self.ncells, (out.size, self.ncells)
        return out

    def unpack(self, packed: np.ndarray):
        return [packed[self.offsets[k]:self.offsets[k + 1]] for k in range(len(self.n_cells))]

    def set_field(self, fid: int, packed: np.ndarray):
        a = np.ascontiguousarray(packed, dtype=np.float64).reshape(-1)
        assert a.size == self.ncells
        self._check(self.be.fn["ensemble_set_field"](self.h, fid, a.ctypes.data, 0))

    def get_field(self, fid: int) -> np.ndarray:
        a = np.empty(self.ncells)
        self._check(self.be.fn["ensemble_get_field"](self.h, fid, a.ctypes.data, 0))
        return a

    def run(self, t_end: float, max_steps: int = 0, block_size: int = 0):
        """Returns (times, steps, device_ms)."""
        k = len(self.n_cells)
        t = (C.c_double * k)()
        s = (C.c_int * k)()
        ms = C.c_double()
        self._check(self.be.fn["ensemble_run"](self.h, t_end, max_steps, block_size, t, s, C.byref(ms)))
        return np.array(t[:]), np.array(s[:]), ms.value

    def autotune(self, probe_steps: int = 20) -> int:
        bs = C.c_int()
        self._check(self.be.fn["ensemble_autotune"](self.h, probe_steps, C.byref(bs)))
        return bs.value


class Context:
    """One solver instance (a SolutionState + solver) in a backend."""

    def __init__(self, be: Backend, handle: C.c_void_p, cfg: Config, mesh: MeshSpec):
        self.be, self.h, self.cfg, self.mesh = be, handle, cfg, mesh
        nx, ny, nz = C.c_int(), C.c_int(), C.c_int()
        self._check(be.fn["extents"](handle, C.byref(nx), C.byref(ny), C.byref(nz)))
        self.shape = (nz.value, ny.value, nx.value)       # numpy (k, j, i), x fastest
        self.ncells = nx.value * ny.value * nz.value
        self.ng = cfg.nGhost

    def _check(self, st: int) -> int:
        if st < 0:
            raise AbiError(st, self.be.error(self.h))
        return st

    def close(self):
        if self.h:
            self.be.fn["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, fid: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert a.size == self.ncells, (a.size, self.ncells)
        self._check(self.be.fn["set_field"](self.h, fid, a.ctypes.data_as(C.c_void_p), 0))

    def get_field(self, fid: int) -> np.ndarray:
        out = np.empty(self.ncells, dtype=np.float64)
        self._check(self.be.fn["get_field"](self.h, fid, out.ctypes.data_as(C.c_void_p), 0))
        return out.reshape(self.shape)

    def set_state(self, fields: dict):
        for fid, arr in fields.items():
            self.set_field(fid, arr)

    def step(self, step: int, time: float, target_dt: float = -1.0) -> float:
        dt = C.c_double()
        self._check(self.be.fn["step"](self.h, step, time, target_dt, C.byref(dt)))
        return dt.value

    def autotune(self, reps: int = 5) -> int:
        """sifv_autotune: the work-unit shape of the 2D fused stage; returns
        the units per warp chosen (0: nothing to tune)."""
        ch = C.c_int()
        self._check(self.be.fn["autotune"](self.h, reps, C.byref(ch)))
        return ch.value

    def set_work_units(self, units_per_warp: int):
        """sifv_set_work_units: fix the work-unit shape of the 2D fused stage."""
        self._check(self.be.fn["set_work_units"](self.h, units_per_warp))

    def set_comm(self, exchange, allreduce_min, allreduce_max=None):
        """Halo exchange and reductions of a decomposed run (sifv_set_comm):
        exchange(pointers, stream) gets the field addresses (ints) the
        step asks to exchange; allreduce_min / allreduce_max(pointer, stream)
        the address of the device (or host) double to reduce (the time step;
        the pressure solvers' residual).  Each returns None or 0; an
        exception is reported to the library as a failure."""
        def ex(user, fields, n, stream):
            try:
                r = exchange([fields[q] for q in range(n)], stream)
                return int(r or 0)
            except Exception:   # a Python error must not cross the C boundary
                import traceback
                traceback.print_exc()
                return 1

        def reducer(fn):
            def red(user, value, stream):
                try:
                    return int(fn(value, stream) or 0)
                except Exception:
                    import traceback
                    traceback.print_exc()
                    return 1
            return ALLREDUCE_MIN_FN(red)
        mx = reducer(allreduce_max) if allreduce_max is not None else ALLREDUCE_MIN_FN()
        self._comm_cb = (EXCHANGE_FN(ex), reducer(allreduce_min), mx)   # kept alive with the context
        c = Comm(self._comm_cb[0], self._comm_cb[1], None, self._comm_cb[2])
        self._check(self.be.fn["set_comm"](self.h, C.byref(c)))

    def set_immersed_bodies(self, bodies):
        """ImmersedBoundaryMethod::addBody for each body + classifyCells."""
        arr = (IbBody * max(len(bodies), 1))(*bodies)
        self._check(self.be.fn["set_immersed_bodies"](self.h, arr, len(bodies)))

    def ib_cell_types(self) -> np.ndarray:
        out = np.empty(self.ncells, dtype=np.uint8)
        self._check(self.be.fn["ib_cell_types"](self.h, out.ctypes.data_as(C.c_void_p)))
        return out.reshape(self.shape)

    def apply_ib_ghost_cells(self):
        self._check(self.be.fn["apply_ib_ghost_cells"](self.h))

    def check_nan(self):
        """(SIFV_F_* id, interior cell) of the first NaN, or (-1, -1)."""
        f, c = C.c_int(), C.c_longlong()
        self._check(self.be.fn["check_nan"](self.h, C.byref(f), C.byref(c)))
        return f.value, c.value

    def run_time_loop(self, end_time: float, output_interval: float, vtk: Optional[VtkSession] = None,
                      print_interval: int = 1, check_nan: bool = True, step0: int = 0, batch: int = 0,
                      progress=None):
        """runTimeLoop on this context; returns (status, LoopResult).
        progress(step, time, dt) is called at the printed steps."""
        p = TimeLoop(end_time, output_interval, print_interval, int(check_nan), step0, batch)
        r = LoopResult()
        cb = PROGRESS_FN(lambda _u, s, t, dt: progress(s, t, dt)) if progress else PROGRESS_FN()
        st = self.be.fn["run_time_loop"](self.h, C.byref(p), vtk.h if vtk else None, cb, None, C.byref(r))
        if st < 0 and st != ERR_NAN:
            raise AbiError(st, self.be.error(self.h))
        return st, r

    def reference_time_loop(self, directory: str, base: str, end_time: float, output_interval: float,
                            print_interval: int = 1) -> int:
        """The reference's own runTimeLoop + VTKSession (reference backend only)."""
        n = C.c_int()
        self._check(self.be.fn["reference_time_loop"](self.h, directory.encode(), base.encode(), end_time,
                                                      output_interval, print_interval, C.byref(n)))
        return n.value

    def advance(self, step0: int, time0: float, t_end: float, n_steps: int):
        t, n = C.c_double(), C.c_int()
        self._check(self.be.fn["advance"](self.h, step0, time0, t_end, n_steps, C.byref(t), C.byref(n)))
        return t.value, n.value

    # ---- discrete adjoint / tangent (explicit single-phase FP64 step) ----
    @staticmethod
    def _sched(schedule):
        if schedule is None:
            return None, 0, None
        a = np.ascontiguousarray(schedule, dtype=np.float64)
        return a.ctypes.data_as(C.POINTER(C.c_double)), a.size, a

    def adjoint_forward(self, step0: int, time0: float, t_end: float, max_steps: int = 0, every: int = 32,
                        schedule=None):
        """Forward run recording the dt sequence and checkpoints; returns (time, steps)."""
        p, n, keep = self._sched(schedule)
        t, k = C.c_double(), C.c_int()
        self._check(self.be.fn["adjoint_forward"](self.h, step0, time0, t_end, max_steps, every, p, n,
                                                  C.byref(t), C.byref(k)))
        return t.value, k.value

    def adjoint_set_precision(self, precision: int):
        """PREC_FP64 or PREC_MIXED (FP32 local Jacobians in the reverse sweep)."""
        self._check(self.be.fn["adjoint_set_precision"](self.h, precision))

    def adjoint_schedule(self) -> np.ndarray:
        n = C.c_int()
        self._check(self.be.fn["adjoint_schedule"](self.h, None, 0, C.byref(n)))
        out = np.empty(n.value)
        self._check(self.be.fn["adjoint_schedule"](self.h, out.ctypes.data_as(C.POINTER(C.c_double)), n.value,
                                                   C.byref(n)))
        return out

    def adjoint_set_seed(self, fid: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert a.size == self.ncells
        self._check(self.be.fn["adjoint_set_seed"](self.h, fid, a.ctypes.data, 0))

    def adjoint_backward(self) -> float:
        ms = C.c_double()
        self._check(self.be.fn["adjoint_backward"](self.h, C.byref(ms)))
        return ms.value

    def adjoint_get_gradient(self, fid: int) -> np.ndarray:
        out = np.empty(self.ncells)
        self._check(self.be.fn["adjoint_get_gradient"](self.h, fid, out.ctypes.data, 0))
        return out.reshape(self.shape)

    def tangent_set_direction(self, fid: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert a.size == self.ncells
        self._check(self.be.fn["tangent_set_direction"](self.h, fid, a.ctypes.data, 0))

    def tangent_forward(self, step0: int, time0: float, t_end: float, max_steps: int = 0, schedule=None):
        p, n, keep = self._sched(schedule)
        t, k = C.c_double(), C.c_int()
        self._check(self.be.fn["tangent_forward"](self.h, step0, time0, t_end, max_steps, p, n,
                                                  C.byref(t), C.byref(k)))
        return t.value, k.value

    def tangent_get(self, fid: int) -> np.ndarray:
        out = np.empty(self.ncells)
        self._check(self.be.fn["tangent_get"](self.h, fid, out.ctypes.data, 0))
        return out.reshape(self.shape)

    def last_pressure_iterations(self) -> int:
        it = C.c_int()
        self._check(self.be.fn["last_pressure_iterations"](self.h, C.byref(it)))
        return it.value

    def pressure_solve(self, rho, rhoc2, rhs, p, dt, tol, max_iter):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, rhoc2, rhs)]
        pp = np.array(p, dtype=np.float64).reshape(-1)
        it = C.c_int()
        st = self._check(self.be.fn["pressure_solve"](
            self.h, *[a.ctypes.data_as(C.c_void_p) for a in arrs], pp.ctypes.data_as(C.c_void_p),
            dt, tol, max_iter, 0, C.byref(it)))
        return pp.reshape(self.shape), it.value, st

    def igr_solve(self, step: int):
        self._check(self.be.fn["igr_solve"](self.h, step))

    def acoustic_dt(self, cfl: float, max_dt: float) -> float:
        d = C.c_double()
        self._check(self.be.fn["acoustic_dt"](self.h, cfl, max_dt, C.byref(d)))
        return d.value

    def advective_dt(self, cfl: float, max_dt: float) -> float:
        d = C.c_double()
        self._check(self.be.fn["advective_dt"](self.h, cfl, max_dt, C.byref(d)))
        return d.value

    def convert_cons_to_prim(self):
        self._check(self.be.fn["convert_cons_to_prim"](self.h))

    def apply_bc(self):
        self._check(self.be.fn["apply_bc"](self.h))

    def set_pressure_solver(self, kind: int):
        self._check(self.be.fn["set_pressure_solver"](self.h, kind))

    def last_step_stats(self):
        ms, n = C.c_double(), C.c_int()
        self._check(self.be.fn["last_step_stats"](self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def profile_step(self, step: int, time: float, target_dt: float = -1.0):
        """Per-kernel-family device time of one step: {family: (ms, launches)}."""
        names = C.create_string_buffer(4096)
        ms = (C.c_double * 64)()
        cnt = (C.c_int * 64)()
        n = C.c_int()
        self._check(self.be.fn["profile_step"](self.h, step, time, target_dt, names, 4096, ms, cnt, 64,
                                               C.byref(n)))
        fams = names.value.decode().split("\n") if n.value else []
        return {f: (ms[k], cnt[k]) for k, f in enumerate(fams)}

    def interior_slices(self):
        """(k, j, i) slices of the physical cells."""
        d = self.cfg.dim
        g = self.ng
        gj = g if d >= 2 else 0
        gk = g if d >= 3 else 0
        nz, ny, nx = self.shape
        return slice(gk, nz - gk), slice(gj, ny - gj), slice(g, nx - g)

    def interior(self, arr: np.ndarray) -> np.ndarray:
        """Slice the physical cells out of a (k, j, i) field."""
        return arr[self.interior_slices()]
