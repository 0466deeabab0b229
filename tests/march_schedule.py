"""A CPU model of the schedule of the 2D wavefront sweep kernel k_march_gs
(semiimplicitfv_b200/csrc/sifv_gs_march.cuh), for tests only.

It restates the kernel's per-lane logic step by step: the skewed pair
layout and every pointer / window of its loads (bounds-checked), the
register rings of prefetched pairs and edge pairs (a load reads memory at
its issue step), shuffles between lanes, the shared-memory edge ring, the
ghost-lane redirects, every wait of the batch and sweep starts, the buffer
rotation and the convergence rule.  Groups (warps) run as generators that
yield at each wait and, at random, after publishing a batch's progress,
interleaved in a random order, so a wait that does not cover a dependency
shows up as a wrong value.  Slots the kernel never
writes hold NaN.  `ref_gs` / `ref_igr` are the plain in-place sweeps
(GaussSeidelPressureSolver::solve, src/GaussSeidelPressureSolver.cpp:60-100;
IGR, src/IGR.cpp:110-156, 2D) with one ghost layer; Python floats are IEEE
doubles without fused multiply-adds, like the kernels' FP64 arithmetic
(compiled with --fmad=false), and their correctly rounded division equals
the kernels' Markstein quotients.
"""
import random

import numpy as np

RE = 256
FIN = 0x7fffffff
NAN = float('nan')


def ref_igr(nx, ny, bc, cf, s0, iters):
    """IGR sweeps in place: ghosts as stored for sweep 0, filled from the interior after each sweep."""
    p = s0.copy()   # (ny + 2, nx + 2) with the stored ghost layer
    for it in range(iters):
        for j in range(ny):
            for i in range(nx):
                rflx, rfrx, rfly, rfry, ax, ay, rh, de = (cf[k][j, i] for k in range(8))
                off = 0.0
                off += ax * (p[j + 1, i] / rflx + p[j + 1, i + 2] / rfrx)
                off += ay * (p[j, i + 1] / rfly + p[j + 2, i + 1] / rfry)
                p[j + 1, i + 1] = (rh + off) / de
        p[1:-1, 0] = p[1:-1, nx] if bc[0] else p[1:-1, 1]
        p[1:-1, nx + 1] = p[1:-1, 1] if bc[1] else p[1:-1, nx]
        p[0, 1:-1] = p[ny, 1:-1] if bc[2] else p[1, 1:-1]
        p[ny + 1, 1:-1] = p[1, 1:-1] if bc[3] else p[ny, 1:-1]
    return p
FIN = 0x7fffffff
NAN = float('nan')


def ref_gs(nx, ny, bc, cf, p0, tol, maxIter):
    p = np.zeros((ny + 2, nx + 2))
    p[1:-1, 1:-1] = p0
    it_done = maxIter
    prev = None
    for it in range(maxIter):
        p[1:-1, 0] = p[1:-1, nx] if bc[0] else p[1:-1, 1]
        p[1:-1, nx + 1] = p[1:-1, 1] if bc[1] else p[1:-1, nx]
        p[0, 1:-1] = p[ny, 1:-1] if bc[2] else p[1, 1:-1]
        p[ny + 1, 1:-1] = p[1, 1:-1] if bc[3] else p[ny, 1:-1]
        prev = p.copy()
        mr = 0.0
        for j in range(ny):
            for i in range(nx):
                c0, c1, c2, c3, co, de, rh = (cf[k][j, i] for k in range(7))
                od = 0.0
                od += c0 * p[j + 1, i] + c1 * p[j + 1, i + 2]
                od += c2 * p[j, i + 1] + c3 * p[j + 2, i + 1]
                pn = (rh + co * od) / de
                r = abs(pn - p[j + 1, i + 1])
                p[j + 1, i + 1] = pn
                mr = mr if mr >= r else r
        if mr < tol:
            it_done = it + 1
            break
    return p, prev, it_done


def emulate(pnx, pny, pbc, cf, p0, tol, maxIter, nb, seed, tr=False, D=8, W=2, KIND=0, S=1):
    """Run the schedule (S segments along the march axis); returns (the
    result with one ghost layer, the iteration count)."""
    rng = random.Random(seed)
    # march space: m along the walk, n across the lanes
    nx, ny = (pny, pnx) if tr else (pnx, pny)
    bc = (pbc[2], pbc[3], pbc[0], pbc[1]) if tr else pbc
    def phys(m, n):   # (x, y) of march cell (m, n)
        return (n, m) if tr else (m, n)
    NH = (nx + 1) // 2
    SW = NH + 32
    G, GA = ny // 32 + 1, (ny + 1) // 32 + 1
    Lseg = (NH + S - 1) // S
    S = (NH + Lseg - 1) // Lseg

    def seg_steps(s):
        return min(NH, (s + 1) * Lseg) - s * Lseg + 31
    ctas = (G + W - 1) // W
    qn = GA * SW * 32

    def mq(g, s, b):
        return (g * SW + s) * 32 + b

    def srcx(i):
        if i < 0: return nx - 1 if bc[0] else 0
        if i >= nx: return 0 if bc[1] else nx - 1
        return i

    def srcy(j):
        if j < 0: return ny - 1 if bc[2] else 0
        if j >= ny: return 0 if bc[3] else ny - 1
        return j

    Q = [np.full((qn, 2), NAN) for _ in range(nb)]
    rec = np.full((qn * 8, 2), NAN)
    igrRec = {}
    for g in range(GA):
        for s in range(SW):
            for b in range(32):
                h, j = s - b, 32 * g + b - 1
                if KIND == 1 and h >= 0 and 2 * h < nx and -1 <= j <= ny:
                    for e in range(2):
                        x = 2 * h + e
                        if x >= nx: break
                        X, Y = phys(x, j)
                        Q[0][mq(g, s, b), e] = p0[Y + 1, X + 1]   # p0 holds the stored ghost layer
                        if 0 <= j < ny:
                            igrRec[(mq(g, s, b), e)] = tuple(cf[k][Y, X] for k in range(8))
                    continue
                if 0 <= j < ny and h >= 0 and 2 * h < nx:
                    for e in range(2):
                        x = 2 * h + e
                        if x >= nx: break
                        X, Y = phys(x, j)
                        Q[0][mq(g, s, b), e] = p0[Y, X]
                        base = ((g * SW + s) * 8 + 4 * e) * 32 + b
                        rec[base] = (cf[0][Y, X], cf[1][Y, X])
                        rec[base + 32] = (cf[2][Y, X], cf[3][Y, X])
                        rec[base + 64] = (cf[4][Y, X], cf[5][Y, X])
                        rec[base + 96] = (1.0 / cf[5][Y, X], cf[6][Y, X])

    def LD(arr, idx):   # bounds-checked load of a pair
        assert 0 <= idx < len(arr), ("OOB load", idx, len(arr))
        return tuple(arr[idx])

    prog = [0] * G
    done = [0] * maxIter
    res = [0.0] * maxIter
    flags = [0, 0]
    sp = {(s, g): (0 if g < G else FIN) for s in range(S) for g in range(ctas * W)}
    eRing = {(s, w): [(NAN, NAN)] * RE for s in range(S) for w in range(ctas * W)}
    nWarps = G * S
    xsLo = nx - 1 if bc[0] else 0
    xsHi = 0 if bc[1] else nx - 1
    perLoY, perHiY = bc[2], bc[3]

    def igr_cell(act, r, pL, pR, pD, pU):
        if not act: return 1.0
        xm, xp, ym, yp = (pD, pU, pL, pR) if tr else (pL, pR, pD, pU)
        rflx, rfrx, rfly, rfry, ax, ay, rh, de = r
        off = 0.0
        off += ax * (xm / rflx + xp / rfrx)
        off += ay * (ym / rfly + yp / rfry)
        return (rh + off) / de

    def cell(act, c0, c1, c2, c3, pL, pR, pD, pU):
        xm, xp, ym, yp = (pD, pU, pL, pR) if tr else (pL, pR, pD, pU)
        od = 0.0
        od += c0[0] * xm + c0[1] * xp
        od += c1[0] * ym + c1[1] * yp
        num = c3[1] + c2[0] * od if act else 1.0
        dv = c2[1] if act else 1.0
        return num / dv

    def group(g, seg):
        c, warp = g // W, g % W
        hs0, hs1 = seg * Lseg, min(NH, (seg + 1) * Lseg)
        nP = hs1 - hs0
        NS = nP + 31
        gLo = c * W - 1 if c > 0 else -1
        topR = ny
        topG, topB = topR >> 5, topR & 31
        gT, bT = (ny + 1) >> 5, (ny + 1) & 31
        hasAbove = g + 1 < G
        L = {}
        for lane in range(32):
            d = {}
            r = 32 * g + lane
            d['rowIn'] = 1 <= r <= ny
            d['low'] = g == 0 and lane == 0
            d['top'] = g == gT and lane == bT and bT >= 1
            d['tAct0'] = lane if d['rowIn'] else NS
            d['tAct1'] = lane + nP if d['rowIn'] else NS
            hLastX = (nx - 1) >> 1
            d['tLast'] = lane + hLastX - hs0 if hs0 <= hLastX < hs1 else -1
            ek, elo, ehi = 0, 0, 0
            if lane == 0 and warp == 0 and g > 0: ek, ehi = 1, nP
            elif d['low'] and perLoY: ek, ehi = 2, nP
            elif lane == 31 and hasAbove: ek, elo, ehi = 3, 31, nP + 31
            elif lane == 31 and g + 1 == gT and bT == 0: ek, elo, ehi = 4, 31, nP + 31
            d['ek'], d['elo'], d['ehi'] = ek, elo, ehi
            d['pLo'] = (max(0, bT - 1) if perHiY else 1) if d['top'] else 0
            d['eWriter'] = lane == 31 and warp < W - 1 and d['rowIn']
            L[lane] = d
        lastOdd = ((nx - 1) & 1) != 0
        chk = 0

        inCta0 = g - 1 >= c * W
        inCta1 = g + 1 < c * W + W
        inCta2 = c * W <= topG < c * W + W
        extG = [(g - 1) if (g > 0 and not inCta0) else -1, (g + 1) if (hasAbove and not inCta1) else -1,
                topG if (g == 0 and perLoY and topG != 0 and not inCta2) else -1]

        def progress_of(h):
            if c * W <= h < c * W + W:
                return sp[(seg, h)]
            if h in extG:
                return sp[(seg, h)]
            return -1

        for k in range(maxIter):
            base, prevBase = k * NS, (k - 1) * NS
            kw = k + 1 - nb
            if flags[0]: break
            while True:
                a = kw < 0 or done[kw] >= nWarps
                b = not (perHiY and g == G - 1 and g != 0) or sp[(seg, 0)] >= base
                sl = seg == 0 or sp[(seg - 1, g)] >= (k + 1) * seg_steps(seg - 1)
                sr = seg == S - 1 or k == 0 or sp[(seg + 1, g)] >= (k - 1) * seg_steps(seg + 1) + 32
                if a and b and sl and sr: break
                if flags[0]: break
                yield
            if flags[0]: break
            go = True
            while KIND == 0 and go and chk < k:
                if done[chk] < nWarps: break
                if res[chk] < tol:
                    flags[0] = 1
                    go = False
                chk += 1
            if not go or flags[0]: break
            Qk, Qn = Q[k % nb], Q[(k + 1) % nb]
            rowK = {lane: mq(g, 0, lane) for lane in range(32)}
            rowKs = {lane: mq(g, hs0, lane) for lane in range(32)}
            stored0 = KIND == 1 and k == 0
            lowFromEdge = perLoY and not stored0
            pP, eP, pLoK = {}, {}, {}
            for lane in range(32):
                d = L[lane]
                p = rowKs[lane]
                pLoK[lane] = 0 if stored0 else d['pLo']
                if not stored0:
                    if d['low'] and not perLoY: p = mq(0, hs0 + 1, 1)
                    if d['top']:
                        p = (mq(0, hs0 + 1, 1) - 32 * bT) if perHiY else (mq(gT, hs0, bT - 1) - 32)
                pP[lane] = p
                ek = d['ek']
                if ek == 1: e = ('n', mq(g - 1, hs0 + 31, 31))
                elif ek == 2: e = ('k', mq(topG, hs0 + topB, topB))
                elif ek == 3: e = ('k', mq(g + 1, hs0, 0) - 32 * 31)
                elif ek == 4:
                    if stored0: e = ('k', mq(g + 1, hs0, 0) - 32 * 31)
                    else: e = ('k', (mq(0, hs0 + 1, 1) - 32 * 31) if perHiY else rowKs[lane])
                else: e = ('k', rowKs[lane])
                eP[lane] = e
            gL, gR = {}, {}
            for lane in range(32):
                if hs0 > 0:   # a later segment starts from the left segment's new last cell
                    gL[lane] = LD(Qn, mq(g, hs0 - 1 + lane, lane))[1]
                    gR[lane] = NAN
                    if L[lane]['tLast'] >= 0 and L[lane]['rowIn']:
                        if stored0:
                            n_ = 32 * g + lane - 1
                            XR, YR = phys(nx, n_)
                            gR[lane] = p0[YR + 1, XR + 1]
                        else:
                            gR[lane] = LD(Qk, rowK[lane] + 32 * ((xsHi >> 1) + lane))[xsHi & 1]
                    continue
                if stored0:
                    n_ = 32 * g + lane - 1 if L[lane]['rowIn'] else 0
                    XL, YL = phys(-1, n_)
                    XR, YR = phys(nx, n_)
                    gL[lane] = p0[YL + 1, XL + 1]
                    gR[lane] = p0[YR + 1, XR + 1]
                    continue
                a = LD(Qk, rowK[lane] + 32 * ((xsLo >> 1) + lane)) if L[lane]['rowIn'] else (NAN, NAN)
                bq = LD(Qk, rowK[lane] + 32 * ((xsHi >> 1) + lane)) if L[lane]['rowIn'] else (NAN, NAN)
                gL[lane] = a[xsLo & 1]
                gR[lane] = bq[xsHi & 1]
            eOff = base & (RE - 1)

            def batch_wait(tu, tp):
                n0 = base + min(tu + 32, NS) if warp > 0 else -1
                n1 = base + min(tp + 32, NS) if (warp == 0 and g > 0) else -1
                n2 = prevBase + min(tp + topB + 1, NS) if (g == 0 and lowFromEdge and topG != 0) else -1
                n3 = prevBase + min(tp - 30, NS) if (hasAbove and tp - 30 > 0) else -1
                n4 = base + tu - 30 - RE if (warp < W - 1 and hasAbove) else -1

                def met():
                    return ((n0 < 0 or sp[(seg, g - 1)] >= n0) and (n1 < 0 or progress_of(g - 1) >= n1) and
                            (n2 < 0 or progress_of(topG) >= n2) and (n3 < 0 or progress_of(g + 1) >= n3) and
                            (n4 < 0 or sp[(seg, g + 1)] >= n4))
                while not met():
                    if flags[0]: return
                    yield

            def ldE(lane, t):
                kind, base_ = eP[lane]
                arr = Qn if kind == 'n' else Qk
                return LD(arr, base_ + 32 * t)

            yield from batch_wait(-1, D - 1)
            if flags[0]: break
            pr = {lane: [(0.0, 0.0)] * D for lane in range(32)}
            er = {lane: [(0.0, 0.0)] * D for lane in range(32)}
            for u in range(D):
                for lane in range(32):
                    d = L[lane]
                    if u >= pLoK[lane]: pr[lane][u] = LD(Qk, pP[lane] + 32 * u)
                    if d['elo'] <= u < d['ehi']: er[lane][u] = ldE(lane, u)
            newPair = {lane: (0.0, 0.0) for lane in range(32)}
            maxRes = {lane: 0.0 for lane in range(32)}
            aborted = False
            for t0 in range(0, NS, D):
                yield from batch_wait(t0 + D - 1, t0 + 2 * D - 1)
                if flags[0]:
                    aborted = True
                    break
                for u in range(D):
                    t = t0 + u
                    if t >= NS: continue
                    Pt = {l: pr[l][u] for l in range(32)}
                    Pn = {l: pr[l][(u + 1) % D] for l in range(32)}
                    eg = {l: er[l][u] for l in range(32)}
                    tn = t + D
                    for lane in range(32):
                        d = L[lane]
                        # through step NS before another segment: lane 31's last pair reads its first pair
                        if tn < NS + (1 if hs1 < NH else 0) and tn >= pLoK[lane]:
                            pr[lane][u] = LD(Qk, pP[lane] + 32 * tn)
                        if tn < NS and d['elo'] <= tn < d['ehi']: er[lane][u] = ldE(lane, tn)
                    up = {l: newPair[l - 1] if l > 0 else newPair[0] for l in range(32)}
                    down = {l: Pn[l + 1] if l < 31 else Pn[31] for l in range(32)}
                    newNP = dict(newPair)
                    for lane in range(32):
                        d = L[lane]
                        eb = eRing[(seg, g - 1)][(eOff + t) & (RE - 1)] if warp > 0 else (NAN, NAN)
                        if lane == 0:
                            pD = eb if warp > 0 else eg[lane]
                        else:
                            pD = up[lane]
                        pU = eg[lane] if lane == 31 else down[lane]
                        act0 = d['tAct0'] <= t < d['tAct1']
                        act1 = act0 and not (t == d['tLast'] and not lastOdd)
                        base0 = ((g * SW + hs0 + t) * 8) * 32 + lane
                        if act0:
                            a = [tuple(rec[base0 + 32 * q]) for q in range(4)]
                            bb = [tuple(rec[base0 + 32 * (4 + q)]) for q in range(4)]
                        else:
                            a = bb = [(0.0, 0.0)] * 4
                        pL0 = gL.get(lane, NAN) if t == lane else newPair[lane][1]
                        pR0 = gR[lane] if (t == d['tLast'] and not lastOdd) else Pt[lane][1]
                        pR1 = gR[lane] if t == d['tLast'] else Pn[lane][0]
                        if KIND == 1:
                            slot = rowKs[lane] + 32 * t
                            pn0 = igr_cell(act0, igrRec.get((slot, 0)), pL0, pR0, pD[0], pU[0])
                            pn1 = igr_cell(act1, igrRec.get((slot, 1)), pn0, pR1, pD[1], pU[1])
                        else:
                            pn0 = cell(act0, *a, pL0, pR0, pD[0], pU[0])
                            pn1 = cell(act1, *bb, pn0, pR1, pD[1], pU[1])
                        if act0:
                            r0 = abs(pn0 - Pt[lane][0])
                            maxRes[lane] = maxRes[lane] if maxRes[lane] >= r0 else r0
                        if act1:
                            r1 = abs(pn1 - Pt[lane][1])
                            maxRes[lane] = maxRes[lane] if maxRes[lane] >= r1 else r1
                        if act0:
                            idx = rowKs[lane] + 32 * t
                            assert 0 <= idx < qn
                            Qn[idx] = (pn0, pn1 if act1 else 1.0)
                            if d['eWriter']:
                                eRing[(seg, g)][(eOff + t - 31) & (RE - 1)] = (pn0, pn1 if act1 else 1.0)
                            newNP[lane] = (pn0, pn1 if act1 else 1.0)
                        elif d['low']:
                            newNP[lane] = eg[lane] if lowFromEdge else Pt[lane]
                    newPair = newNP
                sp[(seg, g)] = base + min(t0 + D, NS)
                if rng.random() < 0.5:   # other warps may see every published progress value
                    yield
            if aborted: break
            v = 0.0
            for lane in range(32):
                m = maxRes[lane]
                m = 0.0 if m != m else m
                v = v if v >= m else m
            res[k] = max(res[k], v)
            done[k] += 1
            yield
        sp[(seg, g)] = FIN

    gens = {(s, g): group(g, s) for s in range(S) for g in range(G)}
    alive = set(gens)
    steps = 0
    while alive:
        g = rng.choice(sorted(alive))
        for _ in range(rng.randint(1, 6)):
            try:
                next(gens[g])
            except StopIteration:
                alive.discard(g)
                break
        steps += 1
        if steps > 20_000_000:
            raise RuntimeError("no progress")
    iters = maxIter
    for jj in range(maxIter if KIND == 0 else 0):
        if res[jj] < tol:
            iters = jj + 1
            break
    fin, prv = Q[iters % nb], Q[(iters - (0 if KIND else 1)) % nb]
    out = np.zeros((pny + 2, pnx + 2))

    def psrc(i, n, lo, hi):
        if i < 0: return n - 1 if lo else 0
        if i >= n: return 0 if hi else n - 1
        return i
    for j in range(-1, pny + 1):
        for i in range(-1, pnx + 1):
            inn = 0 <= i < pnx and 0 <= j < pny
            xs, ys = (i, j) if inn else (psrc(i, pnx, pbc[0], pbc[1]), psrc(j, pny, pbc[2], pbc[3]))
            m, n = (ys, xs) if tr else (xs, ys)
            r = n + 1
            v = (fin if inn else prv)[mq(r >> 5, (m >> 1) + (r & 31), r & 31)]
            out[j + 1, i + 1] = v[m & 1]
    return out, iters
