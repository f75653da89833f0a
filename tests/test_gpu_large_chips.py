"""Chips larger than the kernels' shared memory holds at once: the CUDA-core correlation
streams the chip in column chunks (and the tensor-core path is not eligible beyond 226 rows),
so every chip size the reference accepts runs.

Against the oracle on a few points: integer peaks identical, correlation within 1e-6 (UInt8;
the FP64 chip sums of areas above 4096 round in a different order) or 1e-5 (Float32), sub-pixel
offsets within 1e-3 px except cascade-argmax near-ties.
"""

import numpy as np
import pytest

from conftest import fields

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,chip,r,tol,bf16", [(np.uint8, 256, 24, 1e-6, 1),
                                                   (np.float32, 192, 32, 1e-5, 0),
                                                   (np.float32, 192, 32, 5e-5, 1),
                                                   (np.uint8, 128, 60, 1e-6, 1)])
def test_large_chip_against_oracle(ar, O, gpu_lib, dtype, chip, r, tol, bf16):
    """bf16 = 0: the direct FP32 correlation streams the chip in column chunks; bf16 = 1 (the
    default) runs Float32 on the split-BF16 tensor-core kernel, whose chip operand comes in
    chunks too."""
    ref, sec = ar.synthetic.shifted_pair(768, (2.6, -3.3), seed=31, dtype=dtype)
    rng = np.random.default_rng(chip + r)
    pts = ar.pointset(rng.uniform(330, 440, 6), rng.uniform(330, 440, 6), chip_size=chip,
                      search_radius=r)
    p = ar.params(preprocess="none", quantize="none", upsampling=16)
    ctx = ar._lib.Context(0)
    ctx.set_option(ar._lib.AR_OPT_SPLIT_BF16, bf16)
    d = ar.track(ar.ImagePair(ref, sec), pts, p, ctx=ctx)
    ctx.close()
    dx, dy, cc, searched = O.track(ref, sec, fields(pts), upsampling=16)
    assert np.array_equal(d.searched.ravel(order="F"), searched.astype(bool))
    got = d.correlation.ravel(order="F")
    ok = ~np.isnan(cc)
    assert ok.all() and np.array_equal(np.isnan(got), np.isnan(cc))
    assert np.max(np.abs(got[ok] - cc[ok])) <= tol
    gx, gy = d.dx.ravel(order="F"), d.dy.ravel(order="F")
    assert np.max(np.abs(gx - dx)) <= 1e-3 and np.max(np.abs(gy - dy)) <= 1e-3


def test_chip_64_pipeline_reaches_256(ar, gpu_lib):
    """The default levels of chip_size = 64 are 64, 128 and 256."""
    a, b, v, _ = ar.synthetic.scale_u16_pair(1024, seed=12)
    v[300:700, 300:700] = False  # a large hole: its points fall through to the coarsest level
    r = ar.autorift(a, b, secondary_valid=v, chip_size=64, grid_spacing=32, search_radius=20)
    assert set(np.unique(r.chip_size).tolist()) <= {0, 64, 128, 256}
    assert np.isfinite(r.dx).mean() > 0.5
