"""The block search of the sub-pixel cascade kernel (k_refine), restated in numpy float32 with
the kernel's operation order, against the full cascade.

k_refine materialises levels 1-3, then computes only the 16 x 16 final-level blocks whose bound
can reach the maximum, each through its dependency cone above level 3, and stops when no
remaining bound reaches the best value. This test replays exactly that search (bounds from the
level-3 cone with k * 2^-20 * max|level 2| slack over the L - 3 levels above it, the two-level
bound at level L - 2 when it is above level 3, the region sizes the kernel's buffers hold) on
peaked, random, flat and tied 5 x 5 patches and checks that it returns the full cascade's value
and row-major-first position (src/peak.jl:456-522). The GPU tests check the kernel itself
against the oracle's full cascade.
"""

import numpy as np
import pytest

import numpy as np
f32 = np.float32
def taps(p, n):
    c = p >> 1; q = min(c + 1, n - 1)
    if p & 1: return 2, c, c, q
    m = 1 if c == 0 else c - 1
    return 3, m, c, q
def sample(nt, a, b, c):
    if nt == 3: return f32(f32(f32(0.75) * b) + f32(f32(0.125) * f32(a + c)))
    return f32(f32(0.5) * f32(b + c))
def pyrup_full(src):
    S = src.shape[0]; D = 2 * S
    tmp = np.zeros((D, S), f32)
    for i in range(D):
        nt, m, c, q = taps(i, S)
        for j in range(S): tmp[i, j] = sample(nt, src[m, j], src[c, j], src[q, j])
    dst = np.zeros((D, D), f32)
    for j in range(D):
        nt, m, c, q = taps(j, S)
        for i in range(D): dst[i, j] = sample(nt, tmp[i, m], tmp[i, c], tmp[i, q])
    return dst
def pyrup_fast(src):
    # vectorised, same ops
    S = src.shape[0]; D = 2 * S
    idx = [taps(i, S) for i in range(D)]
    nt = np.array([t[0] for t in idx]); m = np.array([t[1] for t in idx]); c = np.array([t[2] for t in idx]); q = np.array([t[3] for t in idx])
    A, B, C = src[m, :], src[c, :], src[q, :]
    t3 = (f32(0.75) * B).astype(f32) + (f32(0.125) * (A + C).astype(f32)).astype(f32)
    t2 = (f32(0.5) * (B + C).astype(f32)).astype(f32)
    tmp = np.where((nt == 3)[:, None], t3.astype(f32), t2).astype(f32)
    A, B, C = tmp[:, m], tmp[:, c], tmp[:, q]
    t3 = (f32(0.75) * B).astype(f32) + (f32(0.125) * (A + C).astype(f32)).astype(f32)
    t2 = (f32(0.5) * (B + C).astype(f32)).astype(f32)
    return np.where((nt == 3)[None, :], t3.astype(f32), t2).astype(f32)
def full_argmax(P, L):
    cur = P
    for _ in range(L): cur = pyrup_fast(cur)
    n = cur.shape[0]
    flat = cur.reshape(-1)  # row-major index i*n + j
    best = np.nanmax(flat); idx = int(np.flatnonzero(flat == best)[0])
    return best, idx
def tap_range(p0, p1, n):
    lo = (p0 >> 1) if (p0 & 1) else max((p0 >> 1) - 1, 0)
    return lo, min((p1 >> 1) + 1, n - 1)
cap = [16, 10, 7, 6, 5, 5]
def pruned(P, L, stats):
    L1 = pyrup_fast(P); L2 = pyrup_fast(L1); L3 = pyrup_fast(L2)
    amax = f32(np.max(np.abs(L2)))
    ulp = f32(amax * f32(9.5367431640625e-07))
    slack = lambda k: f32(f32(k * ulp) + f32(k * 2.3509887e-38))
    nfinal = 5 << L; nb = nfinal // 16
    def range3(b):
        lo, hi = b * 16, b * 16 + 15
        for lev in range(L - 1, 2, -1):
            lo, hi = tap_range(lo, hi, 5 << lev)
        return lo, hi
    BND = np.zeros(nb * nb, f32)
    for blk in range(nb * nb):
        bi, bj = blk % nb, blk // nb
        r0, r1 = range3(bi); c0, c1 = range3(bj)
        BND[blk] = f32(L3[r0:r1 + 1, c0:c1 + 1].max() + slack(L - 3))
    bv, bi_ = f32(-np.inf), 2**31 - 1
    visited = full = 0
    while True:
        m = BND.max(); sel = int(np.flatnonzero(BND == m)[0])
        if m == -np.inf or m < bv: break
        BND[sel] = -np.inf; visited += 1
        bI, bJ = sel % nb, sel // nb
        cl = [(bI * 16, bI * 16 + 15, bJ * 16, bJ * 16 + 15)]
        for d in range(1, L - 2):
            n = 5 << (L - d)
            r0, r1 = tap_range(cl[-1][0], cl[-1][1], n); c0, c1 = tap_range(cl[-1][2], cl[-1][3], n)
            cl.append((r0, r1, c0, c1))
        for d in range(len(cl)):
            assert cl[d][1] - cl[d][0] + 1 <= cap[d] and cl[d][3] - cl[d][2] + 1 <= cap[d], (d, cl[d])
        # the cone above level 3: region values at each level from the region below, with the
        # same taps (cl[L - 3] is the level-3 region)
        sreg = cl[L - 3]; src = {(i, j): L3[i, j] for i in range(sreg[0], sreg[1] + 1) for j in range(sreg[2], sreg[3] + 1)}
        pr = False
        for d in range(L - 4, -1, -1):
            n = 5 << (L - d - 1)
            r0, r1, c0, c1 = cl[d]
            tmp = {}
            for i in range(r0, r1 + 1):
                nt, mm, cc, qq = taps(i, n)
                for j in range(sreg[2], sreg[3] + 1):
                    tmp[(i, j)] = sample(nt, src[(mm, j)], src[(cc, j)], src[(qq, j)])
            dst = {}
            for j in range(c0, c1 + 1):
                nt, mm, cc, qq = taps(j, n)
                for i in range(r0, r1 + 1):
                    dst[(i, j)] = sample(nt, tmp[(i, mm)], tmp[(i, cc)], tmp[(i, qq)])
            src = dst; sreg = cl[d]
            if d == 2:
                mx = max(dst.values())
                if f32(mx + slack(2)) < bv: pr = True; break
        if pr: continue
        full += 1
        for (i, j), v in src.items():
            idx = i * nfinal + j
            if v > bv or (v == bv and idx < bi_): bv, bi_ = v, idx
    stats.append((visited, full))
    return bv, bi_



def patch(kind, rng):
    if kind == 0:  # a smooth correlation peak with noise
        yy, xx = np.mgrid[0:5, 0:5]
        cy, cx = rng.uniform(1, 3, 2)
        return (0.9 * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / rng.uniform(1, 4))
                + rng.normal(0, 0.01, (5, 5))).astype(f32)
    if kind == 1:
        return rng.uniform(-1, 1, (5, 5)).astype(f32)
    if kind == 2:  # constant: every block ties
        return np.full((5, 5), f32(0.25))
    return rng.choice([f32(0.5), f32(0.5), f32(-0.75)], (5, 5)).astype(f32)  # plateaus


@pytest.mark.parametrize("L", [4, 5, 6])
@pytest.mark.parametrize("kind", [0, 1, 3])
def test_block_search_matches_full_cascade(L, kind):
    rng = np.random.default_rng(10 * L + kind)
    stats = []
    for _ in range(2):
        P = patch(kind, rng)
        got = pruned(P, L, stats)
        want = full_argmax(P, L)
        assert got[0] == want[0] and got[1] == want[1]
    if kind == 0:
        assert max(s[1] for s in stats) < (5 << L) ** 2 // 256  # the search prunes


def test_block_search_constant_patch():
    stats = []
    P = patch(2, None)
    assert pruned(P, 4, stats) == full_argmax(P, 4)
