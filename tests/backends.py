"""Loaders for the libraries the tests compare.

- ``oracle()``: the C restatement (oracle/libsifv_oracle.so, prefix sifvo_)
- ``reference()``: the reference sources built in place with the MPI shim
  (oracle/_ref/libsifv_ref.so, prefix sifvr_), None when not built
- ``cuda()``: the CUDA library of the package (prefix sifv_)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

from semiimplicitfv_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
_cache = {}


def _build_oracle():
    if not os.path.exists(os.path.join(ORACLE_DIR, "libsifv_oracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)


def oracle() -> abi.Backend:
    if "oracle" not in _cache:
        _build_oracle()
        lib = ctypes.CDLL(os.path.join(ORACLE_DIR, "libsifv_oracle.so"))
        _cache["oracle"] = abi.Backend(lib, "sifvo_", "oracle")
    return _cache["oracle"]


def reference(release: bool = False):
    key = "ref_release" if release else "ref"
    if key not in _cache:
        path = os.path.join(ORACLE_DIR, "_ref", "libsifv_ref_release.so" if release else "libsifv_ref.so")
        if not os.path.exists(path):
            # oracle/Makefile builds it where the reference sources are present
            # (SIFV_REFERENCE_DIR overrides its default location), else skips
            ref = os.environ.get("SIFV_REFERENCE_DIR")
            subprocess.run(["make", "-s", "-j8", "-C", ORACLE_DIR, "ref"] + ([f"REF={ref}"] if ref else []),
                           check=True, stdout=subprocess.DEVNULL)
        if not os.path.exists(path):
            _cache[key] = None
        else:
            lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
            _cache[key] = abi.Backend(lib, "sifvr_", "reference-release" if release else "reference")
    return _cache[key]


def cuda() -> abi.Backend:
    if "cuda" not in _cache:
        from semiimplicitfv_b200 import _lib
        _cache["cuda"] = abi.Backend(_lib.load(), "sifv_", "cuda")
    return _cache["cuda"]


def make(backend: abi.Backend, case):
    cfg, mesh, fields = case
    ctx = backend.create(cfg, mesh)
    ctx.set_state(fields)
    return ctx


def mpi_run(backend: abi.Backend, case, nranks: int, warmup: int, steps: int, fids=None, gather: bool = True,
            procs=None, pressure_kind: int = 0):
    """Run the reference's own solver on ``case`` decomposed over ``nranks``
    MPI ranks (threads of this process through the MPI shim):
    ``warmup`` steps, then ``steps`` timed steps; ``procs`` fixes the process
    grid (ranks per axis; None: MPI_Dims_create), ``pressure_kind`` the
    semi-implicit pressure solver (0 Jacobi, 1 Gauss-Seidel).  Returns
    (seconds of the timed steps, max over ranks; the dts of all steps; the
    process grid; {field id: global array} of the final state when
    ``gather``; the pressure iterations of every step)."""
    import numpy as np
    f = backend.lib.sifvr_mpi_run
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(abi.Config), ctypes.POINTER(abi.Mesh), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                  ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    cfg, mesh, fields = case
    fids = list(fields) if fids is None else list(fids)
    init = [np.ascontiguousarray(fields[k], dtype=np.float64) for k in fids]
    out = [np.zeros_like(a) for a in init] if gather else None
    ids = (ctypes.c_int * len(fids))(*fids)
    pin = (ctypes.c_void_p * len(fids))(*[a.ctypes.data for a in init])
    pout = (ctypes.c_void_p * len(fids))(*[a.ctypes.data for a in out]) if gather else None
    sec = ctypes.c_double()
    dts = (ctypes.c_double * max(warmup + steps, 1))()
    iters = (ctypes.c_int * max(warmup + steps, 1))()
    dims = (ctypes.c_int * 3)()
    pr = (ctypes.c_int * 3)(*procs) if procs is not None else None
    ms = mesh.cstruct()
    st = f(ctypes.byref(cfg), ctypes.byref(ms), nranks, pr, pressure_kind, len(fids), ids, pin, pout, warmup, steps,
           ctypes.byref(sec), dts, iters, dims)
    if st != abi.OK:
        raise abi.AbiError(st, backend.error(None))
    return (sec.value, list(dts)[:warmup + steps], tuple(dims), (dict(zip(fids, out)) if gather else None),
            list(iters)[:warmup + steps])
