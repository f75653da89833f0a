"""Host emulations of the index mappings and arithmetic facts the tensor-core kernels rely on.

Each test restates, in numpy, one piece of `csrc/ar_track.cu` or `csrc/ar_prepare.cu` exactly as
the kernel computes it and checks it against the direct definition:

* the Toeplitz product structure of the tensor-core numerators (window blocks of 16 rows, the
  chip operand rows trimmed per block by `block_rows`, accumulator column = surface row) against
  a direct correlation, and that every product writes accumulator columns below round16(nr);
* the striped FP64 box sums of `k_corr_bf` (column sums per stripe, then a running sum along each
  surface row whose differences cw columns apart are the box sums) against direct box sums;
* the three-limb BF16 split: v == l0 + l1 + l2 for normal Float32 v, and two limbs for integers
  below 2^16 in magnitude;
* the flattened order of `k_corr_tc`'s wide-surface epilogue (every value visited once) and the
  ring rows of the carried box sums;
* the integer per-thread partial sums of `staged_chip_stats` against the FP64 running sums they
  replace (bit for bit, within the kernel's bound);
* `k_corr_tc`'s staging task maps (chip blocks and window blocks, each written once) and that the
  carried box sums read only the window blocks the kernel transposed for them;
* the FP32 mean of `k_highpass_w`: the correctly rounded FP32 quotient of an integer sum by a
  count equals the FP64 quotient rounded to FP32 (double rounding innocuous), for every count
  the kernel can see.
"""

import numpy as np
import pytest


def block_rows(q, NB, nr):
    """`block_rows` (csrc/ar_track.cu): operand rows [elo, elo + n) of window block q."""
    lo = max(0, NB - 16 - 16 * q)
    hi = min(NB, NB - 16 + nr - 16 * q)
    if hi <= lo:
        return None
    elo = lo & ~15
    n = (hi - elo + 15) & ~15
    return elo, n


def toeplitz_numerator(W, C, nr, nc):
    """The products as the kernels issue them: for each chip column b and window block q,
    D[j, dcol + e'] += sum_r A[j, r] B[elo + e', r] with A[j, r] = W[16 q + r, j + b] and
    B[e, r] = C[r - u, b], u = e - NB + 16, into accumulator columns dcol = 16 q + elo - NB + 16.
    Returns the surface (nr x nc) read from accumulator columns 0 .. nr - 1 and the largest
    column any product wrote."""
    ch, cw = C.shape
    NB = (ch + 15 + 15) // 16 * 16
    QB = (ch + nr - 1 + 15) // 16
    rows = 16 * QB
    Wp = np.zeros((rows + 16, W.shape[1] + 64))
    Wp[:W.shape[0], :W.shape[1]] = W
    AC = 64 + 16  # room to detect a write past round16(nr)
    D = np.zeros((64, AC))
    top = 0
    for b in range(cw):
        # E_b[e][r] = C[r - u, b], u = e - NB + 16 (zero outside the chip)
        E = np.zeros((NB, 16))
        for e in range(NB):
            u = e - NB + 16
            for r in range(16):
                a = r - u
                if 0 <= a < ch:
                    E[e, r] = C[a, b]
        for q in range(QB):
            br = block_rows(q, NB, nr)
            if br is None:
                continue
            elo, n = br
            dcol = 16 * q + elo - (NB - 16)
            assert dcol >= 0
            A = Wp[16 * q:16 * q + 16, b:b + 64].T  # A[j, r]
            B = E[elo:elo + n]                       # B[e', r]
            D[:, dcol:dcol + n] += A @ B.T
            top = max(top, dcol + n)
    return D[:nc, :nr].T, top


@pytest.mark.parametrize("ch,cw,nr,nc", [(32, 32, 50, 50), (16, 20, 9, 13), (64, 64, 64, 64),
                                         (48, 16, 33, 40), (20, 8, 64, 17), (8, 8, 1, 1)])
def test_toeplitz_products_equal_direct_numerator(ch, cw, nr, nc):
    rng = np.random.default_rng(ch * 131 + nr)
    W = rng.integers(0, 256, (ch + nr - 1, cw + nc - 1)).astype(np.float64)
    C = rng.integers(0, 256, (ch, cw)).astype(np.float64)
    got, top = toeplitz_numerator(W, C, nr, nc)
    want = np.zeros((nr, nc))
    for i in range(nr):
        for j in range(nc):
            want[i, j] = np.sum(C * W[i:i + ch, j:j + cw])
    assert np.array_equal(got, want)
    # Every product stays below round16(nr): the narrowed accumulators (round16(nr) columns).
    assert top <= (nr + 15) // 16 * 16


def striped_box_sums(W, ch, cw, nr, nc, XS, threads=256):
    """k_corr_bf's box sums: stripes of XS window columns; column sums V(i, x) of ch rows by
    (column, row segment) tasks sliding down; then, per surface row and sum, a running sum Q over
    the window columns in order: at column xg < nc the running sum is stashed in S[xg], and at
    column xg = j + cw - 1 the box sum S[j] = Q - stash."""
    XW = cw + nc - 1
    S = np.zeros((2, nc, nr))
    q = np.zeros((nr, 2))
    for x0 in range(0, XW, XS):
        xn = min(XS, XW - x0)
        raw = W[:ch + nr - 1, x0:x0 + xn]
        V = np.zeros((xn, nr, 2))
        segs = max(1, min(nr, threads // xn))
        ln = (nr + segs - 1) // segs
        for t in range(xn * segs):
            x, i0 = t % xn, (t // xn) * ln
            i1 = min(nr, i0 + ln)
            if i0 >= i1:
                continue
            col = raw[:, x]
            h1, h2 = col[i0:i0 + ch].sum(), (col[i0:i0 + ch] ** 2).sum()
            for i in range(i0, i1):
                V[x, i] = (h1, h2)
                if i + 1 < i1:
                    h1 += col[i + ch] - col[i]
                    h2 += col[i + ch] ** 2 - col[i] ** 2
        for i in range(nr):
            for comp in range(2):
                for x in range(xn):
                    xg = x0 + x
                    if xg < nc:
                        S[comp, xg, i] = q[i, comp]
                    q[i, comp] += V[x, i, comp]
                    j = xg - cw + 1
                    if 0 <= j < nc:
                        S[comp, j, i] = q[i, comp] - S[comp, j, i]
    return S


@pytest.mark.parametrize("ch,cw,nr,nc,XS", [(8, 6, 5, 7, 4), (16, 16, 8, 8, 3), (6, 10, 4, 9, 30),
                                            (4, 4, 1, 1, 2), (5, 1, 3, 3, 2), (12, 20, 16, 11, 7)])
def test_striped_box_sums_equal_direct(ch, cw, nr, nc, XS):
    rng = np.random.default_rng(ch + 7 * cw + XS)
    W = rng.integers(0, 65536, (ch + nr - 1, cw + nc - 1)).astype(np.float64)
    S = striped_box_sums(W, ch, cw, nr, nc, XS)
    for j in range(nc):
        for i in range(nr):
            box = W[i:i + ch, j:j + cw]
            assert S[0, j, i] == box.sum() and S[1, j, i] == (box ** 2).sum()


def bf16_rn(x):
    """Float32 -> BF16 (round to nearest even), returned as Float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def split3(v):
    """`bf16_split3`: three limbs, each difference in FP32."""
    v = np.asarray(v, np.float32)
    l0 = bf16_rn(v)
    r1 = (v - l0).astype(np.float32)
    l1 = bf16_rn(r1)
    r2 = (r1 - l1).astype(np.float32)
    l2 = bf16_rn(r2)
    return l0, l1, l2


def test_three_bf16_limbs_are_exact():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(200000).astype(np.float32),
                        (rng.standard_normal(50000) * 1e4).astype(np.float32),
                        (rng.random(50000) * 2 - 1).astype(np.float32) * np.float32(3e-3)])
    l0, l1, l2 = split3(v)
    # Exact: the limbs have at most 8 significant bits each and no overlap.
    back = (l0.astype(np.float64) + l1.astype(np.float64)) + l2.astype(np.float64)
    assert np.array_equal(back, v.astype(np.float64))


def test_integer_window_needs_two_limbs():
    w = np.arange(-65535, 65536, dtype=np.float32)
    l0, l1, l2 = split3(w)
    assert np.all(l2 == 0)
    assert np.array_equal(l0.astype(np.float64) + l1.astype(np.float64), w.astype(np.float64))


def test_fp32_mean_equals_fp64_mean_rounded():
    """k_highpass_w divides in FP32: for integer sums |a| < 2^24 and counts 1..81 the correctly
    rounded FP32 quotient equals the FP64 quotient rounded to FP32."""
    rng = np.random.default_rng(5)
    for cnt in range(1, 82):
        lim = cnt * 65535
        a = np.concatenate([np.arange(-2000, 2001), rng.integers(-lim, lim + 1, 20000)])
        a = a[np.abs(a) < (1 << 24)]
        f32 = a.astype(np.float32) / np.float32(cnt)          # IEEE FP32 division
        f64 = (a.astype(np.float64) / np.float64(cnt)).astype(np.float32)
        assert np.array_equal(f32.view(np.uint32), f64.view(np.uint32)), cnt


def flattened_visits(nr, nc, threads=256, group=4):
    """`k_corr_tc`'s flattened epilogue order: thread t starts at e = t (row e mod nr, column
    e div nr) and steps by `threads`, advancing the row by threads mod nr and the column by
    threads div nr with one carry; `group` values per step, the last ones masked by e < nr nc."""
    ne = nr * nc
    fdj, fdi = threads // nr, threads - (threads // nr) * nr
    seen = np.zeros((nr, nc), np.int64)
    for t in range(threads):
        fj, fi = t // nr, t - (t // nr) * nr
        for e in range(t, ne, group * threads):
            for u in range(group):
                if e + u * threads < ne:
                    assert fi + fj * nr == e + u * threads
                    seen[fi, fj] += 1
                fi += fdi
                fj += fdj
                if fi >= nr:
                    fi -= nr
                    fj += 1
    return seen


@pytest.mark.parametrize("nr,nc", [(66, 66), (94, 94), (80, 81), (1, 128), (256, 64), (300, 3),
                                   (128, 128), (17, 100)])
def test_flattened_epilogue_visits_every_value_once(nr, nc):
    assert np.all(flattened_visits(nr, nc) == 1)


def test_ring_rows_carry_box_sums():
    """Carried box sums: after the held point's sums are shifted up by sh rows (ring base
    advanced by sh, only the last sh rows recomputed), every ring row holds the new point's sums."""
    rng = np.random.default_rng(3)
    ch, cw, nr, nc = 12, 10, 30, 20
    NRS = nr | 1
    W = rng.integers(0, 256, (ch + nr - 1 + 200, cw + nc - 1)).astype(np.int64)

    def box(r0, i, j):
        return W[r0 + i:r0 + i + ch, j:j + cw].sum()

    S = np.zeros((nc, NRS), np.int64)
    rbase, r0 = 0, 0
    ring = lambda i: (i + rbase) % NRS
    for i in range(nr):
        for j in range(nc):
            S[j, ring(i)] = box(r0, i, j)
    for sh in (8, 8, 3, 29, 1, 8):
        r0 += sh
        rbase = (rbase + sh) % NRS
        for i in range(nr - sh, nr):
            for j in range(nc):
                S[j, ring(i)] = box(r0, i, j)
        for i in range(nr):
            for j in range(nc):
                assert S[j, ring(i)] == box(r0, i, j)


def chip_sq_partials(C, bd=256, kUA=16):
    """Per-thread partial sums of squared deviations as the CUDA-core kernel forms them: the FP64
    mean S/nn, then thread t adds fl(fl(v - mean)^2) over elements t, t + bd, ... of the
    column-major chip with rows padded to a multiple of kUA (padding skipped)."""
    ch, cw = C.shape
    nn = ch * cw
    S = float(C.sum())
    mean = S / nn
    chp = (ch + kUA - 1) // kUA * kUA
    part = np.zeros(bd)
    for e in range(chp * cw):
        a, b = e % chp, e // chp
        if a < ch:
            d = float(C[a, b]) - mean
            part[e % bd] = part[e % bd] + d * d
    return part, int(S)


@pytest.mark.parametrize("ch,cw,scale", [(128, 128, 255), (128, 128, 40), (64, 128, 255),
                                         (128, 64, 90), (128, 256, 255)])
def test_integer_chip_partials_equal_fp64_partials(ch, cw, scale):
    """`staged_chip_stats`: for power-of-two areas within its bound, the per-thread partial
    K / nn^2 with K = sum (nn C - S)^2 = nn^2 Q - 2 nn S P + m S^2 in integers is the FP64 running
    sum, bit for bit."""
    rng = np.random.default_rng(ch + cw + scale)
    C = np.clip(rng.normal(128, scale, (ch, cw)), 0, 255).astype(np.int64)
    nn, bd, chp = ch * cw, 256, (ch + 15) // 16 * 16
    terms = (chp * cw + bd - 1) // bd
    exact = terms * (255.0 * nn) ** 2 < 2.0 ** 53
    part, S = chip_sq_partials(C)
    P, Q, m = [0] * bd, [0] * bd, [0] * bd
    for e in range(chp * cw):
        a, b = e % chp, e // chp
        if a < ch:
            v = int(C[a, b])
            P[e % bd] += v
            Q[e % bd] += v * v
            m[e % bd] += 1
    # K = sum (nn C - S)^2 over the thread's elements, from its count, sum and sum of squares.
    K = [nn * nn * Q[t] - 2 * nn * S * P[t] + m[t] * S * S for t in range(bd)]
    assert max(K) < 2 ** 63
    ip = np.array([float(k) / float(nn * nn) for k in K])
    if exact:
        assert np.array_equal(ip.view(np.int64), part.view(np.int64))
    else:
        assert (ch, cw) == (128, 256)  # outside the bound: the kernel keeps the FP64 loop


@pytest.mark.parametrize("ch,nr,delta,sh", [(32, 66, 0, 8), (32, 94, 15, 8), (64, 80, 7, 16),
                                            (16, 88, 3, 1), (128, 50, 9, 8), (32, 66, 4, 65)])
def test_carried_box_sums_read_only_transposed_blocks(ch, nr, delta, sh):
    """`k_corr_tc` with carried box sums transposes only the window blocks q >= qT, qT = (delta +
    iA) / 16 with iA = nr - sh the first recomputed surface row; the column-sum tasks of rows
    iA .. nr - 1 (first sums over ch rows, then a sliding update that reads one row ahead) read
    window rows delta + iA ... delta + nr - 1 + ch, all inside those blocks."""
    iA = nr - sh
    qT = (delta + iA) >> 4
    kBT, XW = 192, 97
    nrw = nr - iA
    nseg = max(1, min((nrw + 7) // 8, kBT // XW))
    seglen = (nrw + nseg - 1) // nseg
    rows = set()
    for seg in range(nseg):
        i0 = iA + seg * seglen
        i1 = min(i0 + seglen, nr)
        if i0 >= i1:
            continue
        rows.update(delta + i0 + a for a in range(ch))   # first sum
        rows.update((delta + i0, delta + i0 + ch))        # outgoing / incoming before the slide
        for i in range(i0, i1 - 1):
            rows.update((delta + i + 1, delta + i + 1 + ch))
    assert min(rows) >= 16 * qT
    # The sums that are carried (rows 0 .. iA - 1) are not recomputed at all.
    assert min(rows) >= delta + iA


@pytest.mark.parametrize("ch,cw", [(32, 32), (17, 9), (128, 128), (64, 31), (226, 4)])
def test_chip_block_tasks_cover_the_chip_once(ch, cw):
    """`k_corr_tc`'s chip staging: task t is 16 rows (block j = t mod nb16) of chip column
    b = t div nb16; two tasks per thread and step. Every row < round16(ch) of every column is
    written once, rows >= ch as zeros (the keep mask)."""
    nb16 = (ch + 15) >> 4
    ntask, bd = nb16 * cw, 256
    written = np.zeros((nb16 * 16, cw), np.int64)
    for tid in range(bd):
        for t0 in range(tid, ntask, 2 * bd):
            for u in range(2):
                t = t0 + u * bd
                if t >= ntask:
                    continue
                b, j = t // nb16, t % nb16
                keep = ch - 16 * j
                for i in range(4):
                    kb = keep - 4 * i
                    nbytes = 4 if kb >= 4 else max(kb, 0)
                    for byte in range(4):
                        r = 16 * j + 4 * i + byte
                        written[r, b] += 1
                        assert (byte < nbytes) == (r < ch)
    assert np.all(written == 1)


@pytest.mark.parametrize("Q,XS", [(7, 160), (12, 192), (1, 96), (10, 130)])
def test_window_block_tasks_cover_each_block_once(Q, XS):
    """`k_corr_tc`'s window staging: task t = (block q = t div XS, column x = t mod XS), three
    tasks per thread and step."""
    bd, ntask = 256, Q * XS
    seen = np.zeros((Q, XS), np.int64)
    for tid in range(bd):
        for t0 in range(tid, ntask, 3 * bd):
            for u in range(3):
                t = t0 + u * bd
                if t < ntask:
                    seen[t // XS, t % XS] += 1
    assert np.all(seen == 1)
