"""The reference's own solver decomposed over MPI ranks (threads of one
process through the MPI shim) -- the form in which the CPU baseline runs the
benchmark grid on every host core.

Checks that the shim's multi-rank MPI (Cartesian decomposition, buffered
halo messages, rank-ordered reductions) reproduces the reference's
single-rank result bit for bit on the explicit step, which exchanges only
ghost copies and reduces dt with an exact minimum: uneven splits, 1D / 2D /
3D process grids, outflow, slip-wall and periodic (self-exchange across the
wrap) faces.  No GPU."""
import numpy as np
import pytest

import backends
import cases
from semiimplicitfv_b200 import abi


def _ref():
    ref = backends.reference()
    if ref is None:
        pytest.skip("reference build absent (oracle/_ref)")
    return ref


CASES = {
    "sod-3ranks": (lambda: cases.sod(200), 3, 10),
    "riemann2d-4ranks": (lambda: cases.riemann2d(64), 4, 5),
    "riemann2d-slipwall-6ranks": (lambda: cases.riemann2d(50, bc=abi.BC_SLIPWALL), 6, 5),
    "riemann2d-periodic-2ranks": (lambda: cases.riemann2d(40, bc=abi.BC_PERIODIC), 2, 5),
    "acoustic3d-periodic-8ranks": (lambda: cases.acoustic3d(12, semi=False, igr=False, rk=3), 8, 3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_decomposed_reference_equals_single_rank(name):
    ref = _ref()
    make, nranks, nsteps = CASES[name]
    single = backends.make(ref, make())
    _, _, dts1 = cases.run_steps(single, nsteps)
    sec, dts, dims, fields, _ = backends.mpi_run(ref, make(), nranks, 0, nsteps)
    assert dims[0] * dims[1] * dims[2] == nranks
    assert dts == dts1
    for fid, arr in fields.items():
        a = single.interior(single.get_field(fid))
        b = single.interior(arr.reshape(single.shape))
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), fid


def test_dims_create_is_balanced():
    ref = _ref()
    # 12 ranks on a 2D grid: MPI_Dims_create gives 4 x 3
    _, _, dims, _, _ = backends.mpi_run(ref, cases.riemann2d(24), 12, 0, 1, gather=False)
    assert dims == (4, 3, 1)
