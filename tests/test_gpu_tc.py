"""The tensor-core operand layouts the UInt8 correlation kernel relies on, checked on the device
through ar_tc_selftest (one tcgen05.mma kind::i8 product of shared-memory operand images).

Each case builds the shared-memory image on the host, states the matrix the descriptor should
see, and compares the accumulator with the integer product computed by numpy.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(ar, a_img, b_img, params):
    ctx = ar._lib.default_context()
    a_img = np.ascontiguousarray(a_img, np.uint8)
    b_img = np.ascontiguousarray(b_img, np.uint8)
    params = list(params) + [0] * (13 - len(params))
    N, nk, dstep = params[9], params[10], params[11]
    out = np.zeros((128, N + (nk - 1) * dstep), np.int32)
    prm = (ctypes.c_int * 13)(*params)
    ctx.check(ctx.lib.ar_tc_selftest(ctx.handle, a_img.ctypes.data, a_img.size, b_img.ctypes.data,
                                     b_img.size, prm, out.ctypes.data))
    return out


def planes(X):
    """K-major SWIZZLE_NONE image of an R x 32 byte matrix: two 16-byte K chunks as planes of R
    rows (LBO = 16 R, SBO = 128)."""
    R = X.shape[0]
    img = np.zeros(2 * R * 16, np.uint8)
    for c in range(2):
        img[c * R * 16:(c + 1) * R * 16] = X[:, 16 * c:16 * c + 16].reshape(-1)
    return img


def lanes(D, M):
    """Accumulator rows from the 128 lanes: M = 64 puts row m in lane (m % 16) + 32 (m // 16)."""
    if M == 128:
        return D
    idx = [(m % 16) + 32 * (m // 16) for m in range(64)]
    return D[idx]


@pytest.mark.parametrize("M,N", [(64, 64), (128, 64), (64, 16), (128, 256)])
def test_plain_product(ar, gpu_lib, M, N):
    rng = np.random.default_rng(M + N)
    A = rng.integers(0, 256, (M, 32), dtype=np.uint8)
    B = rng.integers(0, 256, (N, 32), dtype=np.uint8)
    D = run(ar, planes(A), planes(B), [0, M * 16, 128, 0, 0, N * 16, 128, 0, M, N, 1])
    want = A.astype(np.int64) @ B.astype(np.int64).T
    assert np.array_equal(lanes(D, M)[:, :N], want)


def test_sliding_rows_and_odd_start(ar, gpu_lib):
    """Rows that are successive 16-byte slices of one array (SBO 128, LBO 16), starting at an
    arbitrary row: row m of the operand is bytes [16 (s + m + c), +16) for K chunk c."""
    rng = np.random.default_rng(3)
    T = rng.integers(0, 256, (200, 16), dtype=np.uint8)  # 200 rows of 16 bytes
    M, N, s = 64, 64, 37
    A = np.concatenate([T[s:s + M], T[s + 1:s + 1 + M]], axis=1)
    B = rng.integers(0, 256, (N, 32), dtype=np.uint8)
    D = run(ar, T.reshape(-1), planes(B), [16 * s, 16, 128, 0, 0, N * 16, 128, 0, M, N, 1])
    want = A.astype(np.int64) @ B.astype(np.int64).T
    assert np.array_equal(lanes(D, M)[:, :N], want)


def test_accumulate_over_k_steps(ar, gpu_lib):
    """nk products accumulated, each step advancing both operands (the correlation's loop)."""
    rng = np.random.default_rng(4)
    M, N, nk = 64, 64, 5
    TA = rng.integers(0, 256, (M + 2 * nk + 1, 16), dtype=np.uint8)
    TB = rng.integers(0, 256, (N + 3 * nk + 40, 16), dtype=np.uint8)
    want = np.zeros((M, N), np.int64)
    for st in range(nk):
        A = np.concatenate([TA[2 * st:2 * st + M], TA[2 * st + 1:2 * st + 1 + M]], axis=1)
        # B: K chunk c at LBO = 40 rows; step advances 3 rows.
        B = np.concatenate([TB[3 * st:3 * st + N], TB[3 * st + 40:3 * st + 40 + N]], axis=1)
        want += A.astype(np.int64) @ B.astype(np.int64).T
    D = run(ar, TA.reshape(-1), TB.reshape(-1),
            [0, 16, 128, 32, 0, 40 * 16, 128, 48, M, N, nk])
    assert np.array_equal(lanes(D, M)[:, :N], want)


def test_column_offset_accumulation(ar, gpu_lib):
    """Step s adds into accumulator columns [16 s, 16 s + N): the correlation kernel's compact
    chip operand, whose N rows are the same for every window block."""
    rng = np.random.default_rng(6)
    M, N, nk, dstep = 64, 64, 6, 16
    TA = rng.integers(0, 256, (M + 2 * nk + 1, 16), dtype=np.uint8)
    B = rng.integers(0, 256, (N, 32), dtype=np.uint8)
    want = np.zeros((M, N + (nk - 1) * dstep), np.int64)
    for st in range(nk):
        A = np.concatenate([TA[2 * st:2 * st + M], TA[2 * st + 1:2 * st + 1 + M]], axis=1)
        want[:, st * dstep:st * dstep + N] += A.astype(np.int64) @ B.astype(np.int64).T
    D = run(ar, TA.reshape(-1), planes(B), [0, 16, 128, 32, 0, N * 16, 128, 0, M, N, nk, dstep])
    assert np.array_equal(lanes(D, M), want)


def test_16x256b_read_pattern(ar, gpu_lib):
    """The epilogue's accumulator read: thread t of warp w gets rows 16 w + t // 4 (+ 8) and
    columns 8 k + 2 (t % 4) (+ 1) of the M = 64 accumulator, in registers 4 k + 0..3."""
    rng = np.random.default_rng(8)
    M, N = 64, 64
    A = rng.integers(0, 256, (M, 32), dtype=np.uint8)
    B = rng.integers(0, 256, (N, 32), dtype=np.uint8)
    D = run(ar, planes(A), planes(B), [0, M * 16, 128, 0, 0, N * 16, 128, 0, M, N, 1, 0, 1])
    want = A.astype(np.int64) @ B.astype(np.int64).T
    for w in range(4):
        for t in range(32):
            for k in range(4):
                for v in range(4):
                    row = 16 * w + t // 4 + (8 if v >= 2 else 0)
                    col = 8 * k + 2 * (t % 4) + (v & 1)
                    assert D[32 * w + t, 4 * k + v] == want[row, col], (w, t, k, v)


def test_out_of_image_descriptor_rejected(ar, gpu_lib):
    A = np.zeros(64 * 32, np.uint8)
    B = np.zeros(64 * 32, np.uint8)
    with pytest.raises(ar._lib.ArError):
        run(ar, A, B, [16, 64 * 16, 128, 0, 0, 64 * 16, 128, 0, 64, 64, 1])


def test_bounded_wait_runs_out_and_context_survives(ar, gpu_lib):
    """Failure detection without a fault: a product that is never issued leaves the kernel's
    bounded completion wait to run out; the call reports AR_ERR_TIMEOUT, the kernel returns
    normally, and the same context then computes correctly."""
    ctx = ar._lib.default_context()
    rng = np.random.default_rng(0)
    A = rng.integers(0, 256, (64, 32), dtype=np.uint8)
    B = rng.integers(0, 256, (16, 32), dtype=np.uint8)
    a, b = planes(A), planes(B)
    prm = (ctypes.c_int * 13)(0, 64 * 16, 128, 0, 0, 16 * 16, 128, 0, 64, 16, 1, 0, 2)
    out = np.zeros((128, 16), np.int32)
    rc = ctx.lib.ar_tc_selftest(ctx.handle, a.ctypes.data, a.size, b.ctypes.data, b.size, prm,
                                out.ctypes.data)
    assert rc == 4  # AR_ERR_TIMEOUT
    D = run(ar, a, b, [0, 64 * 16, 128, 0, 0, 16 * 16, 128, 0, 64, 16, 1])
    assert np.array_equal(lanes(D, 64)[:, :16], A.astype(np.int64) @ B.astype(np.int64).T)
    ref, sec = ar.synthetic.shifted_pair(128, (2, 1), dtype=np.uint8)
    d = ar.track(ar.ImagePair(ref, sec), ar.gridpoints(ref.shape, 32, chip_size=16,
                                                        search_radius=6))
    assert np.isfinite(d.dx).all()
