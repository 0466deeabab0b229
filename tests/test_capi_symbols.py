"""The CUDA library loads without a GPU and exports every function that
include/sifv.h declares (no compute calls here)."""
import ctypes
import os
import re

from semiimplicitfv_b200 import _lib, abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "sifv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sifv_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_abi():
    names = _declared()
    for must in ("sifv_create", "sifv_step", "sifv_pressure_solve", "sifv_igr_solve", "sifv_advance",
                 "sifv_pressure_solve_noalloc", "sifv_profile_step"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_binding_matches_library():
    be = abi.Backend(_lib.load(), "sifv_", "cuda")
    assert set(abi._SIGS) <= set(be.fn)


def test_config_validate_without_gpu():
    lib = _lib.load()
    lib.sifv_config_validate.argtypes = [ctypes.POINTER(abi.Config)]
    lib.sifv_last_error.restype = ctypes.c_char_p
    good = abi.config_defaults(dim=2, nGhost=3, reconOrder=abi.WENO5)
    assert lib.sifv_config_validate(ctypes.byref(good)) == abi.OK
    bad = abi.config_defaults(dim=2, nGhost=1, reconOrder=abi.WENO5)
    assert lib.sifv_config_validate(ctypes.byref(bad)) == abi.ERR_BAD_CONFIG
    assert b"nGhost" in lib.sifv_last_error(None)


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    cfg = abi.config_defaults(dim=1, nGhost=3, reconOrder=abi.WENO5)
    mesh = abi.MeshSpec(abi.linspace_nodes(16, 0.0, 1.0))
    be = abi.Backend(_lib.load(), "sifv_", "cuda")
    try:
        be.create(cfg, mesh)
    except abi.AbiError as e:
        assert e.status in (abi.ERR_NO_DEVICE, abi.ERR_CUDA)
    else:
        raise AssertionError("create succeeded without a GPU")


def test_ensemble_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    be = abi.Backend(_lib.load(), "sifv_", "cuda")
    cfg = abi.config_defaults(dim=1, nGhost=3, reconOrder=abi.WENO5)
    try:
        be.create_ensemble(cfg, [16, 32], [0.0, 0.0], [1.0, 2.0])
    except abi.AbiError as e:
        assert e.status in (abi.ERR_NO_DEVICE, abi.ERR_CUDA)
    else:
        raise AssertionError("ensemble create succeeded without a GPU")
    # configuration checks come first and need no device
    bad = abi.config_defaults(dim=2, nGhost=3, reconOrder=abi.WENO5)
    try:
        be.create_ensemble(bad, [16], [0.0], [1.0])
    except abi.AbiError as e:
        assert e.status == abi.ERR_UNSUPPORTED
    else:
        raise AssertionError("2D ensemble accepted")
