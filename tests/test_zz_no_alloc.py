"""The allocation-free Jacobi pressure solve (sifv_pressure_solve_noalloc).

It serves callers that cannot allocate device memory -- a host whose GPU
memory belongs to its own pool allocator, or code that must not call
cudaMalloc/cudaFree between stream operations because those calls can
synchronise the device -- so its scratch lives in a static device array
instead.  This test calls it through the C ABI twice in a row, on different
inputs, and checks each result against the context-based
sifv_pressure_solve with the tolerance of the other parity tests, and
against the oracle's Jacobi solve bit for bit (both CUDA paths evaluate the
reference's expressions in its order), in 1D, 2D and 3D.  It sits in a
file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _noalloc_fn():
    lib = backends.cuda().lib
    f = lib.sifv_pressure_solve_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(abi.Mesh), ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4 + \
                 [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    e = lib.sifv_noalloc_last_error
    e.restype = ctypes.c_char_p
    return f, e


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    return (1.0 + 0.2 * rng.random(n), 1.4 + 0.3 * rng.random(n), rng.random(n), rng.random(n))


CASES = {
    "1d-periodic": lambda: cases.advection1d(96, semi=True),
    "2d-slipwall": lambda: cases.riemann2d(40, bc=abi.BC_SLIPWALL),
    "3d-periodic": lambda: cases.acoustic3d(14),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_noalloc_matches_context_solve_and_oracle_twice(name):
    import torch
    cfg, mesh, fields = CASES[name]()
    ctx = backends.make(backends.cuda(), (cfg, mesh, fields))
    octx = backends.make(backends.oracle(), (cfg, mesh, fields))
    solve, last_error = _noalloc_fn()
    ms = mesh.cstruct()
    n = ctx.ncells
    for call, (seed, dt, max_iter) in enumerate(((1, 1e-2, 40), (2, 3e-2, 25))):
        rho, rhoc2, rhs, p0 = _inputs(n, seed)
        want, want_iters, _ = ctx.pressure_solve(rho, rhoc2, rhs, p0, dt, 1e-12, max_iter)
        ora, ora_iters, _ = octx.pressure_solve(rho, rhoc2, rhs, p0, dt, 1e-12, max_iter)
        dev = [torch.from_numpy(a.copy()).cuda() for a in (rho, rhoc2, rhs, p0)]
        it = ctypes.c_int()
        torch.cuda.synchronize()
        st = solve(ctypes.byref(ms), cfg.dim, cfg.nGhost, *[ctypes.c_void_p(t.data_ptr()) for t in dev],
                   dt, 1e-12, max_iter, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(it))
        assert st >= 0, last_error().decode()
        got = dev[3].cpu().numpy().reshape(ctx.shape)
        assert it.value == want_iters == ora_iters, (call, it.value, want_iters, ora_iters)
        gi, wi = ctx.interior(got), ctx.interior(want)
        rel = np.abs(gi - wi).max() / np.abs(wi).max()
        assert rel <= TOL, (call, rel)
        # bit for bit against the oracle's Jacobi solve
        assert np.array_equal(gi, ctx.interior(ora.reshape(ctx.shape))), call
        # ghost cells are left as the caller passed them
        interior = np.zeros(ctx.shape, dtype=bool)
        ctx.interior(interior)[...] = True
        assert np.array_equal(got[~interior], p0.reshape(ctx.shape)[~interior])


def test_noalloc_rejects_oversize():
    import torch
    solve, last_error = _noalloc_fn()
    x = abi.linspace_nodes(9000, 0.0, 1.0)
    mesh = abi.MeshSpec(x)
    ms = mesh.cstruct()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    it = ctypes.c_int()
    st = solve(ctypes.byref(ms), 1, 3, *[ctypes.c_void_p(t.data_ptr())] * 4, 1e-2, 1e-8, 10, None, ctypes.byref(it))
    assert st == abi.ERR_BAD_ARG
    assert b"SIFV_NOALLOC_MAX_AXIS" in last_error()
