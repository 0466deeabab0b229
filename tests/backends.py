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
            ref_src = "/root/reference/src/ExplicitSolver.cpp"
            if os.path.exists(ref_src):
                subprocess.run(["make", "-s", "-j8", "-C", ORACLE_DIR, "ref"], check=True)
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
