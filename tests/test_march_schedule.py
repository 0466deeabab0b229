"""The schedule of the 2D wavefront sweep kernel (k_march_gs), modelled on the
CPU by tests/march_schedule.py with the groups interleaved at random, gives
the plain in-place sweeps' results bit for bit: Gauss-Seidel iterations
(batch lengths 8 and 4, convergence with speculative sweeps) and IGR sweeps
(stored ghosts read by sweep 0), walking along x or y, periodic and
zero-gradient faces, several CTAs, ghost rows that open a new group, odd and
tiny extents, rows cut into segments along the march axis, and seeded
random configurations of all of these."""
import numpy as np
import pytest

import march_schedule as ms

# (nx, ny, periodic x-, x+, y-, y+)
SHAPES = [(20, 70, (0, 0, 0, 0)), (37, 64, (1, 1, 0, 0)), (19, 95, (0, 0, 1, 1)), (3, 94, (1, 1, 1, 1)),
          (9, 31, (0, 0, 1, 1)), (1, 40, (1, 1, 0, 0))]


def _mask(shape):
    m = np.ones(shape, bool)
    m[0, 0] = m[0, -1] = m[-1, 0] = m[-1, -1] = False   # corners of the one-layer ghost frame
    return m


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}-{''.join(map(str, s[2]))}")
@pytest.mark.parametrize("D,tr", [(8, False), (4, True)])
def test_gauss_seidel_schedule(shape, D, tr):
    nx, ny, bc = shape
    rs = np.random.default_rng(nx * 1000 + ny)
    cf = [rs.random((ny, nx)) * 0.2 for _ in range(4)] + [np.ones((ny, nx)) * 0.9, 1.0 + rs.random((ny, nx)),
                                                          rs.random((ny, nx))]
    p0 = rs.random((ny, nx))
    for max_iter, tol in ((7, 1e-30), (40, 1e-4)):
        pref, prev, itr = ms.ref_gs(nx, ny, bc, cf, p0, tol, max_iter)
        ref = prev.copy()
        ref[1:-1, 1:-1] = pref[1:-1, 1:-1]   # ghosts as the last fill before the last sweep left them
        out, it = ms.emulate(nx, ny, bc, cf, p0, tol, max_iter, nb=3 + (nx % 3), seed=nx + ny, tr=tr, D=D)
        assert it == itr
        m = _mask(ref.shape)
        assert np.array_equal(out[m].view(np.int64), ref[m].view(np.int64))


@pytest.mark.parametrize("shape", SHAPES[:4], ids=lambda s: f"{s[0]}x{s[1]}-{''.join(map(str, s[2]))}")
@pytest.mark.parametrize("tr", [False, True])
def test_igr_schedule(shape, tr):
    nx, ny, bc = shape
    rs = np.random.default_rng(nx * 1000 + ny + 7)
    cf = [1.0 + rs.random((ny, nx)) for _ in range(4)] + [rs.random((ny, nx)) * 0.3, rs.random((ny, nx)) * 0.3,
                                                          rs.random((ny, nx)), 2.0 + rs.random((ny, nx))]
    s0 = rs.random((ny + 2, nx + 2))   # stored ghost cells that differ from the interior's images
    ref = ms.ref_igr(nx, ny, bc, cf, s0, 4)
    out, _ = ms.emulate(nx, ny, bc, cf, s0, 0.0, 4, nb=4, seed=ny, tr=tr, D=4, KIND=1)
    m = _mask(ref.shape)
    assert np.array_equal(out[m].view(np.int64), ref[m].view(np.int64))


@pytest.mark.parametrize("shape,S", [((20, 70), 2), ((37, 64), 3), ((9, 31), 4), ((41, 127), 2)],
                         ids=lambda v: str(v))
@pytest.mark.parametrize("tr", [False, True])
def test_segment_schedule(shape, S, tr):
    """Rows cut into S segments along the march axis (meshes without a
    periodic face): Gauss-Seidel (batch 8 and 4) and IGR sweeps."""
    nx, ny = shape
    bc = (0, 0, 0, 0)
    rs = np.random.default_rng(nx * 1000 + ny)
    cf = [rs.random((ny, nx)) * 0.2 for _ in range(4)] + [np.ones((ny, nx)) * 0.9, 1.0 + rs.random((ny, nx)),
                                                          rs.random((ny, nx))]
    p0 = rs.random((ny, nx))
    for (max_iter, tol), D in (((7, 1e-30), 8), ((40, 1e-4), 4)):
        pref, prev, itr = ms.ref_gs(nx, ny, bc, cf, p0, tol, max_iter)
        ref = prev.copy()
        ref[1:-1, 1:-1] = pref[1:-1, 1:-1]
        out, it = ms.emulate(nx, ny, bc, cf, p0, tol, max_iter, nb=4, seed=S + nx, tr=tr, D=D, S=S)
        assert it == itr
        m = _mask(ref.shape)
        assert np.array_equal(out[m].view(np.int64), ref[m].view(np.int64))
    cf2 = [1.0 + rs.random((ny, nx)) for _ in range(4)] + [rs.random((ny, nx)) * 0.3, rs.random((ny, nx)) * 0.3,
                                                           rs.random((ny, nx)), 2.0 + rs.random((ny, nx))]
    s0 = rs.random((ny + 2, nx + 2))
    ref = ms.ref_igr(nx, ny, bc, cf2, s0, 4)
    out, _ = ms.emulate(nx, ny, bc, cf2, s0, 0.0, 4, nb=4, seed=ny, tr=tr, D=8, KIND=1, S=S)
    m = _mask(ref.shape)
    assert np.array_equal(out[m].view(np.int64), ref[m].view(np.int64))


def _random_case(i):
    """Configuration i of the randomized schedules: a small mesh, its faces,
    segments (only without a periodic face; from two up to one pair per
    segment), batch length, orientation, cell kind and buffer count (down to
    the minimum of three)."""
    rs = np.random.default_rng(9000 + i)
    nx, ny = int(rs.integers(1, 46)), int(rs.integers(1, 100))
    bc = tuple(int(v) for v in np.repeat(rs.integers(0, 2, 2), 2)) if i % 3 else (0, 0, 0, 0)
    tr = bool(rs.integers(0, 2))
    nh = ((ny if tr else nx) + 1) // 2
    S = 1 if any(bc) else int(rs.choice([1, 2, max(1, nh // 2), nh]))
    return nx, ny, bc, S, int(rs.choice([4, 8])), tr, int(rs.integers(0, 2)), int(rs.integers(3, 7))


@pytest.mark.parametrize("i", range(36))
def test_random_schedules(i):
    """Randomized configurations (seeded): the schedule, including
    one-pair segments and three rotating buffers, still gives the plain
    sweeps' bits and, for Gauss-Seidel, their iteration count."""
    nx, ny, bc, S, D, tr, kind, nb = _random_case(i)
    rs = np.random.default_rng(i)
    m = _mask((ny + 2, nx + 2))
    if kind == 0:
        cf = [rs.random((ny, nx)) * 0.2 for _ in range(4)] + [np.ones((ny, nx)) * 0.9, 1.0 + rs.random((ny, nx)),
                                                              rs.random((ny, nx))]
        p0 = rs.random((ny, nx))
        max_iter, tol = (9, 1e-30) if i % 2 else (30, 1e-3)
        pref, prev, itr = ms.ref_gs(nx, ny, bc, cf, p0, tol, max_iter)
        ref = prev.copy()
        ref[1:-1, 1:-1] = pref[1:-1, 1:-1]
        out, it = ms.emulate(nx, ny, bc, cf, p0, tol, max_iter, nb=nb, seed=i, tr=tr, D=D, S=S)
        assert it == itr
    else:
        cf = [1.0 + rs.random((ny, nx)) for _ in range(4)] + [rs.random((ny, nx)) * 0.3, rs.random((ny, nx)) * 0.3,
                                                              rs.random((ny, nx)), 2.0 + rs.random((ny, nx))]
        s0 = rs.random((ny + 2, nx + 2))
        ref = ms.ref_igr(nx, ny, bc, cf, s0, 5)
        out, _ = ms.emulate(nx, ny, bc, cf, s0, 0.0, 5, nb=nb, seed=i, tr=tr, D=D, KIND=1, S=S)
    assert np.array_equal(out[m].view(np.int64), ref[m].view(np.int64)), (nx, ny, bc, S, D, tr, kind, nb)
