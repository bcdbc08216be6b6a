"""The render without allocations (trt_render_noalloc): the entry point for callers that may not call cudaMalloc,
such as a process whose device memory all belongs to one pool allocator, or a plugin host that forbids allocation in
its render callback. The caller's own device buffers go in through the C ABI, and two calls in a row must give what
the allocating entry point (trt_render) gives on the same scene. This file sorts last so that a run stopping at its
first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

from threert_b200 import _native as N
from threert_b200 import prep, scenes

pytestmark = pytest.mark.gpu


def device_desc(P, torch):
    """The scene's buffers copied into device memory the caller (here torch) owns, and their descriptor."""
    keep = [torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()
            for a in (P.vertices, P.leaves, P.nodes, P.tables, P.words, P.env_half)]
    d = N.SceneDesc(keep[0].data_ptr(), keep[0].numel(), keep[1].data_ptr(), keep[1].numel(), keep[2].data_ptr(),
                    keep[2].numel(), keep[3].data_ptr(), keep[3].numel(), keep[4].data_ptr(), keep[4].numel(),
                    keep[5].data_ptr(), P.env_w, P.env_h)
    return d, keep


def test_no_alloc_render_matches_the_allocating_render(gpu):
    torch = pytest.importorskip("torch")
    L = N.lib()
    P = prep.prepare(scenes.cornell(64, 64))
    spp = 8
    want = gpu.upload(P).render_raw(P.params, spp)[0]
    d, keep = device_desc(P, torch)
    accum = torch.zeros(64 * 64 * N.PIXEL_FLOATS, dtype=torch.float32, device="cuda")
    params = np.ascontiguousarray(P.params, dtype=np.uint32)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rc = L.trt_render_noalloc(C.byref(d), params.ctypes.data_as(C.POINTER(C.c_uint32)), 0, spp, 0,
                                  accum.data_ptr(), stream, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        got = accum.cpu().numpy().reshape(-1, N.PIXEL_FLOATS)
        # The same kernels on the same inputs: equal to the allocating render's accum, call after call.
        assert np.allclose(got, want, rtol=1e-6, atol=1e-7), f"call {call}"


def test_no_alloc_render_refuses_an_image_past_its_array(gpu):
    torch = pytest.importorskip("torch")
    L = N.lib()
    P = prep.prepare(scenes.cornell(16, 16))
    d, keep = device_desc(P, torch)
    big = prep.params_with(P.params, width=512, height=512)
    accum = torch.zeros(16, dtype=torch.float32, device="cuda")
    err = C.create_string_buffer(256)
    rc = L.trt_render_noalloc(C.byref(d), big.ctypes.data_as(C.POINTER(C.c_uint32)), 0, 1, 0, accum.data_ptr(),
                              torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 1 and b"too large" in err.value
    # A size whose 32-bit slot count would wrap to zero (2^20 x 2^14 pixels) is refused the same way.
    huge = prep.params_with(P.params, width=1 << 20, height=1 << 14)
    rc = L.trt_render_noalloc(C.byref(d), huge.ctypes.data_as(C.POINTER(C.c_uint32)), 0, 1, 0, accum.data_ptr(),
                              torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 1 and b"too large" in err.value
