"""The allocation-free track entry point (ar_track_device_static) against ar_track_device.

ar_track_device_static is for callers that cannot allocate device memory when they
correlate; it keeps the pass's scratch in a static device array of the library instead of
context-owned buffers. This file checks, through the C ABI, that two calls in a row give the
same dx, dy, correlation and searched as the context-based entry point on the same device
inputs (bit-identical: the same kernels run on the same data), for UInt8 (tensor-core
correlation) and UInt16 (CUDA-core correlation) images; that the calls allocate nothing (the
library's scratch-allocation counter and the device's free memory are unchanged across them);
and that point sets beyond the array's capacity are rejected. It sets up everything it needs,
so it runs alone in a fresh process as well as after the other tests; it is named to be
collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_points(torch, ar, pts, dev):
    cols = {f: torch.from_numpy(pts.flat(f)).to(dev) for f in ar.points.FIELDS}
    st = ar._lib.ArPoints(*(cols[f].data_ptr() for f in ar.points.FIELDS), len(pts))
    return st, cols


def _outputs(torch, n, dev):
    return [torch.full((n,), 7.0, dtype=torch.float32, device=dev) for _ in range(3)] + [
        torch.full((n,), 9, dtype=torch.uint8, device=dev)]


def _run_context(ar, ctx, pair_handle, st, up, outs, stream):
    ctx.check(ctx.lib.ar_track_device(ctx.handle, pair_handle, ctypes.byref(st), up,
                                      ar._lib.AR_ZNCC, *(o.data_ptr() for o in outs),
                                      ctypes.c_void_p(stream)))


def _run_static(ar, lib, dref, dsec, dvalid, shape, dtype, st, up, outs, stream):
    err = ctypes.create_string_buffer(256)
    rc = lib.ar_track_device_static(dref.data_ptr(), dsec.data_ptr(), dvalid.data_ptr(),
                                    shape[0], shape[1], dtype, ctypes.byref(st), up,
                                    ar._lib.AR_ZNCC, *(o.data_ptr() for o in outs),
                                    ctypes.c_void_p(stream), err, 256)
    assert rc == 0, err.value.decode()


def _allocations(lib):
    n = ctypes.c_int64(-1)
    assert lib.ar_scratch_allocations(ctypes.byref(n)) == 0
    return n.value


@pytest.mark.parametrize("np_dtype", [np.uint8, np.uint16])
def test_static_scratch_matches_context_entry_point_twice(ar, np_dtype):
    import torch

    import __graft_entry__ as ge

    ge._load_build_ext().build()
    lib = ar._lib.load()
    ctx = ar._lib.Context(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    code = ar._lib.AR_U8 if np_dtype == np.uint8 else ar._lib.AR_U16
    ref, sec = ar.synthetic.shifted_pair(320, (4.4, -2.7), seed=41, dtype=np_dtype)
    rv = np.ones(ref.shape, bool)
    rv[40:90, 200:260] = False
    pair = ar.ImagePair(ref, sec, rv, None)
    dp = pair.device(ctx)
    # The same images and combined mask as device buffers owned by the caller.
    dref = torch.from_numpy(np.asfortranarray(ref).ravel(order="F")).to(dev)
    dsec = torch.from_numpy(np.asfortranarray(sec).ravel(order="F")).to(dev)
    dvalid = torch.from_numpy(np.asfortranarray(pair.valid()).ravel(order="F").astype(np.uint8)).to(dev)

    cases = [
        (ar.gridpoints(ref.shape, 12, chip_size=32, search_radius=12), 16),
        (ar.pointset(np.linspace(-3, 330, 500), np.linspace(5, 300, 500), chip_size=32,
                     search_radius=10, dx_prior=2.0), 64),
    ]
    with torch.cuda.stream(stream):
        for pts, up in cases:
            st, keep = _device_points(torch, ar, pts, dev)
            want = _outputs(torch, len(pts), dev)
            _run_context(ar, ctx, dp.handle, st, up, want, stream.cuda_stream)
            got = [_outputs(torch, len(pts), dev) for _ in range(2)]
            stream.synchronize()
            # The first static call on this device looks the array's address up; every call
            # after it must leave both the counter and the device's free memory unchanged.
            _run_static(ar, lib, dref, dsec, dvalid, ref.shape, code, st, up, got[0],
                        stream.cuda_stream)
            allocs = _allocations(lib)
            free0 = torch.cuda.mem_get_info(dev)[0]
            for call in range(2):  # calls in a row share the static scratch
                _run_static(ar, lib, dref, dsec, dvalid, ref.shape, code, st, up, got[call],
                            stream.cuda_stream)
                stream.synchronize()
                for g, w, name in zip(got[call], want, ("dx", "dy", "correlation", "searched")):
                    a, b = g.cpu().numpy(), w.cpu().numpy()
                    same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
                    assert same.all(), f"call {call}, {name}: {np.count_nonzero(~same)} differ"
                assert bool(got[call][3].any())
            assert _allocations(lib) == allocs, "the static entry point allocated scratch"
            assert torch.cuda.mem_get_info(dev)[0] == free0, "device free memory changed"


def test_static_scratch_rejects_oversized_point_sets(ar):
    import torch

    import __graft_entry__ as ge

    ge._load_build_ext().build()
    lib = ar._lib.load()
    n = 32769
    st = ar._lib.ArPoints(1, 1, 1, 1, 1, 1, 1, 1, n)  # never dereferenced: rejected first
    err = ctypes.create_string_buffer(256)
    rc = lib.ar_track_device_static(1, 1, 1, 64, 64, ar._lib.AR_U8, ctypes.byref(st), 16,
                                    ar._lib.AR_ZNCC, 1, 1, 1, 1, None, err, 256)
    assert rc == ar._lib.AR_ERR_SIZE
    assert b"32768" in err.value
