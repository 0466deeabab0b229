"""The drop-in C++ adapters (semiimplicitfv_b200/host/SifvCudaSolvers.hpp)
driven side by side with the reference's own solver classes, compiled
against the reference headers (oracle/_ref/libsifv_adapter_selftest.so):

- CudaExplicitSolver vs ExplicitSolver (2D Riemann, all boundary kinds);
- CudaSemiImplicitSolver vs SemiImplicitSolver + JacobiPressureSolver
  (3D periodic pulse with IGR);
- the reference SemiImplicitSolver with CudaJacobiPressureSolver plugged
  into its PressureSolver slot vs the same solver with the reference Jacobi.

The reference-ordered FP64 path must agree bit for bit (0.0)."""
import ctypes
import os

import pytest

from semiimplicitfv_b200 import _lib, abi

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SELFTEST = os.path.join(ROOT, "oracle", "_ref", "libsifv_adapter_selftest.so")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(SELFTEST):
        pytest.skip("adapter self-test library not built (needs the reference sources)")
    ctypes.CDLL(_lib.LIB_PATH, mode=ctypes.RTLD_GLOBAL)
    L = ctypes.CDLL(SELFTEST)
    L.sifv_adapter_selftest_explicit.restype = ctypes.c_double
    L.sifv_adapter_selftest_explicit.argtypes = [ctypes.c_int] * 4
    L.sifv_adapter_selftest_semi.restype = ctypes.c_double
    L.sifv_adapter_selftest_semi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    return L


@pytest.mark.parametrize("bc", [abi.BC_OUTFLOW, abi.BC_PERIODIC, abi.BC_SLIPWALL, abi.BC_SYMMETRY])
def test_explicit_adapter_bit_identical(lib, bc):
    assert lib.sifv_adapter_selftest_explicit(40, 12, abi.PREC_FP64, bc) == 0.0


def test_explicit_adapter_fast_fp64_within_tolerance(lib):
    r = lib.sifv_adapter_selftest_explicit(40, 12, abi.PREC_FP64_FAST, abi.BC_OUTFLOW)
    assert 0.0 <= r <= 1e-10


def test_semi_implicit_adapter_bit_identical(lib):
    it = ctypes.c_int()
    assert lib.sifv_adapter_selftest_semi(12, 3, 0, ctypes.byref(it)) == 0.0
    assert it.value > 0


def test_pressure_solver_plugin_in_reference_solver(lib):
    it = ctypes.c_int()
    assert lib.sifv_adapter_selftest_semi(12, 3, 1, ctypes.byref(it)) == 0.0
    assert it.value > 0


@pytest.mark.parametrize("plugin", [2, 3])
def test_gauss_seidel_adapters_bit_identical(lib, plugin):
    """CudaSemiImplicitSolver given a GaussSeidelPressureSolver (2), and
    CudaGaussSeidelPressureSolver plugged into the reference's own
    SemiImplicitSolver (3), against the reference with Gauss-Seidel."""
    it = ctypes.c_int()
    assert lib.sifv_adapter_selftest_semi(12, 3, plugin, ctypes.byref(it)) == 0.0
    assert it.value > 0


@pytest.mark.parametrize("bc", [abi.BC_NOSLIPWALL, abi.BC_PERIODIC])
def test_explicit_adapter_viscous_bit_identical(lib, bc):
    """viscousParams.mu carried through the adapter into the CUDA step."""
    lib.sifv_adapter_selftest_explicit_viscous.restype = ctypes.c_double
    lib.sifv_adapter_selftest_explicit_viscous.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    assert lib.sifv_adapter_selftest_explicit_viscous(40, 8, bc, 0.01) == 0.0


@pytest.mark.parametrize("slip,igr", [(0, 0), (1, 0), (0, 1)])
def test_explicit_adapter_immersed_boundary_bit_identical(lib, slip, igr):
    """CudaExplicitSolver + CudaImmersedBoundary against ExplicitSolver +
    ImmersedBoundaryMethod with the same IBCircle."""
    lib.sifv_adapter_selftest_ibm.restype = ctypes.c_double
    lib.sifv_adapter_selftest_ibm.argtypes = [ctypes.c_int] * 4
    assert lib.sifv_adapter_selftest_ibm(48, 6, slip, igr) == 0.0
