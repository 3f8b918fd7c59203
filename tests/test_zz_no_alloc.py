"""The allocation-free blur entry point, through the C ABI (gpu).

spkx_gaussian_noalloc serves callers that may not allocate device memory from inside their render
callback (their memory is budgeted by the host application's own allocator, or cudaMalloc's latency and
synchronisation are not allowed there): they pass device buffers and the blur's intermediate planes
come from a fixed scratch array inside the library. This test gives it device buffers it allocated
itself (through torch) and checks two calls in a row against the allocating entry point, spkx_gaussian,
within the tolerances the other blur tests use: separate and in-place buffers, buffers that start off a
16-byte boundary, and a recursive channel
beside channels of zero sigma, which must come back unchanged. It runs last (file name) so that a failure here never
stops the rest of the suite, and it passes alone in a fresh process as well.
"""

import ctypes

import numpy as np
import pytest

from conftest import sc

pytestmark = pytest.mark.gpu

NOALLOC = (ctypes.c_int32, [sc.FP, sc.FP, ctypes.c_uint32, ctypes.c_uint32, sc.DP, ctypes.c_void_p])


def allocating_blur(lib, plane, sigma):
    h, w, _ = plane.shape
    out = np.zeros_like(plane)
    lib.check(lib.lib.spkx_gaussian(plane.ctypes.data_as(sc.FP), out.ctypes.data_as(sc.FP), w, h,
                                    (ctypes.c_double * 3)(*sigma)))
    return out


def test_noalloc_matches_allocating_entry_point(lib):
    import torch

    fn = lib.lib.spkx_gaussian_noalloc
    fn.restype, fn.argtypes = NOALLOC
    rng = np.random.default_rng(42)
    stream = torch.cuda.Stream()
    # (0, 8, 0): a recursive channel beside two channels that no pass may change; in_place: out == in;
    # shift: the buffers start 4 bytes past a 16-byte boundary (the recursive channels then take the
    # one-thread-per-line kernels instead of the block-parallel ones)
    cases = [((300, 257), (0.65, 1.5, 2.9), False, 0), ((480, 640), (3.0, 20.0, 120.0), False, 0),
             ((61, 97), (2.5, 8.0, 0.0), False, 0), ((200, 150), (0.0, 8.0, 0.0), False, 0),
             ((300, 257), (0.65, 1.5, 2.9), True, 0), ((480, 640), (3.0, 20.0, 120.0), True, 0),
             ((120, 90), (0.0, 8.0, 0.0), True, 0), ((480, 640), (3.0, 20.0, 120.0), False, 1),
             ((61, 97), (2.5, 8.0, 0.0), True, 1), ((64, 48), (8.0, 8.0, 8.0), False, 1)]
    for (h, w), sigma, in_place, shift in cases:
        for call in range(2):  # two calls in a row share the scratch array
            plane = (rng.random((h, w, 3), dtype=np.float32) + 0.1 * (call + 1)).astype(np.float32)
            n = h * w * 3
            d_in = torch.empty(n + shift, device="cuda")[shift:].view(h, w, 3)
            d_in.copy_(torch.from_numpy(plane))
            d_out = d_in if in_place else torch.empty(n + shift, device="cuda")[shift:].view(h, w, 3)
            st = fn(ctypes.cast(d_in.data_ptr(), sc.FP), ctypes.cast(d_out.data_ptr(), sc.FP), w, h,
                    (ctypes.c_double * 3)(*sigma), ctypes.c_void_p(stream.cuda_stream))
            assert st == sc.SPK_OK, lib.last_error()
            stream.synchronize()
            got = d_out.cpu().numpy()
            want = allocating_blur(lib, plane, sigma)
            rel = np.abs(got - want) / np.abs(want)
            for c in range(3):
                tol = 1e-5 if sigma[c] >= 3 else 2e-6
                assert rel[..., c].max() <= tol, (h, w, sigma, in_place, call, c, rel[..., c].max())
                if sigma[c] == 0.0:
                    assert np.array_equal(got[..., c], plane[..., c]), (h, w, sigma, in_place, call, c)


def test_noalloc_refuses_frames_beyond_its_scratch(lib):
    fn = lib.lib.spkx_gaussian_noalloc
    fn.restype, fn.argtypes = NOALLOC
    dummy = ctypes.cast(ctypes.c_void_p(16), sc.FP)  # never dereferenced: the size check comes first
    st = fn(dummy, dummy, 1024, 1024, (ctypes.c_double * 3)(1.0, 1.0, 1.0), None)
    assert st == sc.SPK_ERR_INVALID_ARG
    assert "scratch" in lib.last_error()
