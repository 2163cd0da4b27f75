"""Film grain without allocation: av1b_apply_film_grain_noalloc.

Some callers cannot allocate device memory at the point where they need a
frame's film grain - a display callback that re-shows a reference slot (which
holds the picture before grain) under a real-time deadline, where
cudaMalloc / cudaFree may synchronize the whole device, or a host application
that fixes its device memory at start-up. This entry point serves them: the
caller passes the input picture and its own output planes, and the call
allocates nothing; its scratch is a fixed device array shared by every call.

The test runs it through the C ABI on the stored (pre-grain) pictures of two
decoded frames, one call after the other and then the first again, and checks
each output against the film grain output the decoder itself produced for
that frame. The arithmetic is integer, so the tolerance is zero.
"""
import ctypes
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(av1b):
    lib = av1b.lib()
    f = lib.av1b_apply_film_grain_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return lib


def test_noalloc_film_grain_matches_decoder(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    import torch
    lib = _bind(av1b)
    dec = av1b.Decoder(0)
    # 480x270 10-bit, every tool, film grain on every frame
    blobs = [av1b.synth_frame(2, 4, 2024, k) for k in range(3)]
    slots, decoded = [], []
    for k, b in enumerate(blobs):
        d = b.get_refs()
        b.set_refs([slots[k - x] for x in d])
        slot, planes = dec.decode(b)
        b.set_refs(d)
        slots.append(slot)
        decoded.append(planes)
    assert blobs[0].header[3] == 10

    def apply(frame):
        """The entry point on frame `frame`'s stored picture; returns its output planes."""
        w, _, h, _, sx, sy = blobs[frame].header
        shapes = av1b.plane_shapes(w, h, sx, sy)
        src = (ctypes.c_void_p * 3)()
        src_stride = (ctypes.c_int32 * 3)()
        # an older slot reads as the picture before film grain
        assert lib.av1b_slot_planes_device(dec.h, slots[frame], src, src_stride) == 0
        outs = [torch.empty(s, dtype=torch.int16, device='cuda:0') for s in shapes]
        dst = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in outs])
        dst_stride = (ctypes.c_int32 * 3)(*[s[1] for s in shapes])
        view = ctypes.create_string_buffer(4096)
        assert lib.av1b_syntax_view(blobs[frame].ptr, blobs[frame].size, view) == 0
        rc = lib.av1b_apply_film_grain_noalloc(view, src, src_stride, dst, dst_stride, None)
        assert rc == 0
        torch.cuda.synchronize()
        return [t.cpu().numpy().view(np.uint16) for t in outs]

    # two calls in a row on different frames (different grain parameters), then
    # the first frame again: the shared scratch carries nothing over
    for frame in (0, 1, 0):
        got = apply(frame)
        for p in range(3):
            assert np.array_equal(got[p], decoded[frame][p]), 'frame %d plane %d' % (frame, p)

    # sizes beyond the stated maximum are refused
    view = ctypes.create_string_buffer(4096)
    assert lib.av1b_syntax_view(blobs[0].ptr, blobs[0].size, view) == 0
    struct.pack_into('<i', view, 0, 20000)  # width
    src = (ctypes.c_void_p * 3)(1, 1, 1)
    stride = (ctypes.c_int32 * 3)(20000, 20000, 20000)
    assert lib.av1b_apply_film_grain_noalloc(view, src, stride, src, stride, None) == -1
    for s in slots:
        dec.release_reference(s)
    dec.close()
