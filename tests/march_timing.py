"""A timing model of the 2D wavefront sweep kernel k_march_gs
(semiimplicitfv_b200/csrc/sifv_gs_march.cuh) at batch granularity, for tests
only.

Each warp (segment s, row group g) runs its sweeps in order, a batch of D
steps at a time, one time unit per step.  The waits are the kernel's:

- sweep start: the left segment finished this sweep, the right segment did
  the first 32 steps of the previous one, and every warp finished the sweep
  that last used this sweep's output buffer (nb buffers in rotation);
- before a batch: the group below is 32 steps ahead of what the next batch
  reads (inside a CTA the batch being computed, across CTAs the next one,
  whose prefetch reads it), and the group above did the previous sweep up
  to 30 steps short of it;
- across a periodic row axis: the top group starts a sweep after group 0
  finished the previous one, and group 0's batches follow the top row's
  previous sweep.

A warp's progress is seen by warps of its own CTA at once and by others
`delta` units after its batch ends (the helper warp's relay).  The model
holds the step time fixed, so it shows what the waits alone allow.
`buffers` restates the host's choice of nb (march_run in
semiimplicitfv_b200/csrc/sifv_capi.cu).
"""


def segments(NH, S):
    """Segment length and count as the host rounds them."""
    L = (NH + S - 1) // S
    return L, (NH + L - 1) // L


def buffers(NH, G, GA, S, D):
    """Iterate buffers of a launch: the warps' spread in sweeps plus slack,
    at most 32, at most 1 GiB together or 8 buffers where 1 GiB holds
    fewer, at least 3."""
    L, S = segments(NH, S)
    NSs = L + 31
    nb = min(32, 4 + (G * (32 + 2 * D + 40) + S * NSs + NSs - 1) // NSs)
    buf = GA * (NH + 32) * 32 * 16
    return max(3, min(nb, max(1 << 30, 8 * buf) // buf))


def run(NH, G, S, sweeps, D=8, nb=32, delta=4.0, W=2, wrap=None):
    """Times at which all warps finished each sweep (list, in steps).
    wrap = (group, lane) of the last interior row when the row axis is
    periodic (one segment): the top group then starts a sweep after group 0
    finished the previous one (its ghost row above), and group 0 reads its
    ghost row below from that row's previous sweep."""
    L, S = segments(NH, S)

    def steps(s):
        return min(NH, (s + 1) * L) - s * L + 31
    end, pubs, done = {}, {}, []

    def seen(s, g, k, step, same_cta):
        for p, t in pubs[(s, g, k)]:
            if p >= step:
                return t + (0.0 if same_cta else delta)
        raise AssertionError("progress never reaches the step waited for")

    # every wait points to an earlier sweep, or to the same sweep of a lower segment or group
    for k in range(sweeps):
        for s in range(S):
            for g in range(G):
                t = end.get((s, g, k - 1), 0.0)
                if s > 0:
                    t = max(t, end[(s - 1, g, k)] + delta)
                if s < S - 1 and k > 0:
                    t = max(t, seen(s + 1, g, k - 1, 32, False))
                if k + 1 - nb >= 0:
                    t = max(t, done[k + 1 - nb] + delta)
                if wrap and g == G - 1 and g != 0 and k > 0:
                    t = max(t, end[(s, 0, k - 1)] + delta)
                ns, lst = steps(s), []
                for t0 in range(0, ns, D):
                    tp = t0 + 2 * D - 1
                    if g > 0:
                        same = (g - 1) // W == g // W
                        t = max(t, seen(s, g - 1, k, min((t0 + D - 1 if same else tp) + 32, ns), same))
                    if g < G - 1 and k > 0 and tp - 30 > 0:
                        same = (g + 1) // W == g // W
                        t = max(t, seen(s, g + 1, k - 1, min(tp - 30, ns), same))
                    if wrap and g == 0 and k > 0 and wrap[0] != 0:
                        same = wrap[0] // W == 0
                        t = max(t, seen(s, wrap[0], k - 1, min(tp + wrap[1] + 1, ns), same))
                    t += min(D, ns - t0)
                    lst.append((min(t0 + D, ns), t))
                pubs[(s, g, k)] = lst
                end[(s, g, k)] = t
        done.append(max(end[(s, g, k)] for s in range(S) for g in range(G)))
    return done
