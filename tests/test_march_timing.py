"""The iterate buffers the host gives the 2D wavefront (march_run in
semiimplicitfv_b200/csrc/sifv_capi.cu) never hold its pipeline back in the
timing model of tests/march_timing.py: with them, the model's period per
iteration equals the one with unlimited buffers, from 1024² to 8192² and
with rows cut into segments, and with every face periodic.  A cap of 1 GiB
alone would leave 3 buffers at 8192² and nearly double the period there."""
import pytest

import march_timing as mt

SMS = 148   # B200 SMs, one CTA of the Gauss-Seidel kernel (batch 8) on each


def plan(nx, ny):
    """The host's launch plan for a mesh without a periodic face: walk along
    the longer axis, 32 rows per warp, two warps per CTA, segments of about
    192 pairs as far as the co-resident CTAs allow."""
    nm, nn = max(nx, ny), min(nx, ny)
    NH, G, GA = (nm + 1) // 2, nn // 32 + 1, (nn + 1) // 32 + 1
    fit = SMS // ((G + 1) // 2)
    S = max(1, min(fit, (NH + 191) // 192))
    return NH, G, GA, mt.segments(NH, S)[1]


def period(done, first, last):
    return (done[last] - done[first]) / (last - first)


@pytest.mark.parametrize("shape", [(1024, 1024), (2048, 2048), (4096, 512), (8192, 8192)], ids=str)
def test_buffers_leave_no_reuse_stall(shape):
    NH, G, GA, S = plan(*shape)
    nb = mt.buffers(NH, G, GA, S, 8)
    sweeps = 10 if G > 100 else 24
    got = period(mt.run(NH, G, S, sweeps, nb=nb), sweeps // 2, sweeps - 1)
    if S == 1:
        assert got == NH + 31, (nb, got)   # one sweep after another, nothing else waits
    else:
        free = period(mt.run(NH, G, S, sweeps, nb=64), sweeps // 2, sweeps - 1)
        assert got == free, (nb, got, free)


def test_one_gib_alone_would_stall_at_8192():
    NH, G, GA, S = plan(8192, 8192)
    assert (S, (1 << 30) // (GA * (NH + 32) * 32 * 16), mt.buffers(NH, G, GA, S, 8)) == (1, 1, 8)
    assert period(mt.run(NH, G, S, 10, nb=3), 5, 9) > 1.5 * (NH + 31)


@pytest.mark.parametrize("n", [1024, 2048])
def test_buffers_leave_no_reuse_stall_periodic_rows(n):
    """Every face periodic (n × n): batch length 4, the period is the climb
    over all row groups, and the buffers the host picks still leave it as
    with unlimited buffers."""
    NH, G, GA = n // 2, n // 32 + 1, (n + 1) // 32 + 1
    assert G * (32 + 2 * 8 + 10) > NH + 31   # the host's rule for the short batch
    nb, wrap = mt.buffers(NH, G, GA, 1, 4), (n // 32, n % 32)
    got = period(mt.run(NH, G, 1, 16, D=4, nb=nb, wrap=wrap), 8, 15)
    free = period(mt.run(NH, G, 1, 16, D=4, nb=64, wrap=wrap), 8, 15)
    assert got == free > 2 * (NH + 31), (nb, got, free)
