"""Film grain without allocation: av1b_apply_film_grain_noalloc.

Some callers cannot allocate device memory at the point where they need a
frame's film grain - a display callback that re-shows a reference slot (which
holds the picture before grain) under a real-time deadline, where
cudaMalloc / cudaFree may synchronize the whole device, or a host application
that fixes its device memory at start-up. This entry point serves them: the
caller passes the input picture and its own output planes, and the call
allocates nothing; its scratch is a fixed device array shared by every call.

The tests run it through the C ABI on the stored (pre-grain) pictures of
decoded frames and compare each output with the film grain output of the
decoder itself and of the oracle (the reference's CPU backend) for the same
frame: two calls in a row on different frames, then the first again; 4:4:4
and 4:2:2 pictures at 8 and 10 bits and a restricted-range identity-matrix
frame (from the real-stream fixtures, with grain parameters planted); the
copy path of a frame without grain; the refusal of overlapping planes; and
that the calls allocate no device memory. The arithmetic is integer, so the
tolerance is zero.
"""
import ctypes
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# byte offsets in a serialized frame: the scalars start after the 48-byte
# header; color_matrix is the tenth int32, the film grain block follows the 34
# int32 scalars before it (av1b_frame_syntax in include/av1b.h)
_SCALARS = 48
_COLOR_MATRIX = _SCALARS + 9 * 4
_GRAIN = _SCALARS + 34 * 4
_GRAIN_BYTES = 188 * 4
_CLIP = _GRAIN + _GRAIN_BYTES - 4


def _bind(av1b):
    lib = av1b.lib()
    f = lib.av1b_apply_film_grain_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return lib


@pytest.fixture(scope='module')
def gpu(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    import torch
    dec = av1b.Decoder(0)
    yield dec, torch, _bind(av1b)
    dec.close()


def _device_free():
    import torch
    free, _total = torch.cuda.mem_get_info(0)
    return free


def _apply(av1b, lib, torch, dec, blob, slot, outs=None, src=None, src_stride=None):
    """The entry point on `slot`'s stored picture (before grain) with `blob`'s
    grain parameters, into fresh device planes (or `outs`). Returns
    (rc, output planes as numpy or None, the torch output tensors)."""
    w, _, h, _, sx, sy = blob.header
    shapes = av1b.plane_shapes(w, h, sx, sy)
    if src is None:
        src = (ctypes.c_void_p * 3)()
        src_stride = (ctypes.c_int32 * 3)()
        assert lib.av1b_slot_planes_device(dec.h, slot, src, src_stride) == 0
        dec.sync()
    if outs is None:
        outs = [torch.empty(s, dtype=torch.int16, device='cuda:0') for s in shapes]
    dst = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in outs])
    dst_stride = (ctypes.c_int32 * 3)(*[t.shape[1] for t in outs])
    view = ctypes.create_string_buffer(4096)
    assert lib.av1b_syntax_view(blob.ptr, blob.size, view) == 0
    rc = lib.av1b_apply_film_grain_noalloc(view, src, src_stride, dst, dst_stride, None)
    torch.cuda.synchronize()
    if rc:
        return rc, None, outs
    return rc, [t.cpu().numpy().view(np.uint16) for t in outs], outs


def test_noalloc_film_grain_matches_decoder_and_oracle(av1b, gpu):
    dec, torch, lib = gpu
    import refdec
    # 480x270 10-bit 4:2:0, every tool, film grain on every frame
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
    oracle = None
    if refdec.available():
        ref = refdec.RefDecoder()
        oracle = []
        st = refdec.Stream(ref)
        for k, b in enumerate(blobs):
            oracle.append(st.decode(k, b)[1])

    # two calls in a row on different frames (different grain parameters), then
    # the first frame again: the shared scratch carries nothing over
    for frame in (0, 1, 0):
        rc, got, _ = _apply(av1b, lib, torch, dec, blobs[frame], slots[frame])
        assert rc == 0
        for p in range(3):
            assert np.array_equal(got[p], decoded[frame][p]), 'frame %d plane %d' % (frame, p)
            if oracle is not None:
                assert np.array_equal(got[p], oracle[frame][p]), 'oracle: frame %d plane %d' % (frame, p)
    # later calls allocate nothing: neither torch's count nor the device's
    # free memory moves across two more calls into the same output planes
    torch.cuda.synchronize()
    outs = [torch.empty(s, dtype=torch.int16, device='cuda:0')
            for s in av1b.plane_shapes(*[blobs[0].header[i] for i in (0, 2, 4, 5)])]
    before = (torch.cuda.memory_allocated(0), _device_free())
    for frame in (1, 0):
        assert _apply(av1b, lib, torch, dec, blobs[frame], slots[frame], outs=outs)[0] == 0
    assert (torch.cuda.memory_allocated(0), _device_free()) == before

    # sizes beyond the stated maximum are refused
    view = ctypes.create_string_buffer(4096)
    assert lib.av1b_syntax_view(blobs[0].ptr, blobs[0].size, view) == 0
    struct.pack_into('<i', view, 0, 20000)  # width
    src = (ctypes.c_void_p * 3)(1, 1, 1)
    stride = (ctypes.c_int32 * 3)(20000, 20000, 20000)
    assert lib.av1b_apply_film_grain_noalloc(view, src, stride, src, stride, None) == -1
    for s in slots:
        dec.release_reference(s)


def test_noalloc_refuses_overlapping_planes(av1b, gpu):
    """In-place grain (an output plane over an input plane) and output planes
    that overlap each other are refused before anything runs."""
    dec, torch, lib = gpu
    b = av1b.synth_frame(2, 8, 5, 0)
    slot, planes = dec.decode(b)
    w, _, h, _, sx, sy = b.header
    shapes = av1b.plane_shapes(w, h, sx, sy)
    pic = [torch.from_numpy(p.astype(np.int16)).cuda() for p in planes]
    src = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in pic])
    src_stride = (ctypes.c_int32 * 3)(*[t.shape[1] for t in pic])
    # dst == src
    rc, _, _ = _apply(av1b, lib, torch, dec, b, slot, outs=pic, src=src, src_stride=src_stride)
    assert rc == -1
    # one output plane inside another
    big = torch.empty(shapes[0], dtype=torch.int16, device='cuda:0')
    outs = [big, big[1:1 + shapes[1][0], :shapes[1][1]], torch.empty(shapes[2], dtype=torch.int16,
                                                                       device='cuda:0')]
    view = ctypes.create_string_buffer(4096)
    assert lib.av1b_syntax_view(b.ptr, b.size, view) == 0
    dst = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in outs])
    dst_stride = (ctypes.c_int32 * 3)(shapes[0][1], shapes[0][1], shapes[2][1])
    assert lib.av1b_apply_film_grain_noalloc(view, src, src_stride, dst, dst_stride, None) == -1
    # separate planes are accepted
    rc, got, _ = _apply(av1b, lib, torch, dec, b, slot, src=src, src_stride=src_stride)
    assert rc == 0
    dec.release_reference(slot)


def test_noalloc_copies_without_grain(av1b, gpu):
    """A frame without grain (apply == 0): the output is the input."""
    dec, torch, lib = gpu
    b = av1b.synth_frame(1, 8, 5, 0)   # config 1: no film grain
    raw = bytearray(b.to_bytes())
    assert struct.unpack_from('<i', raw, _GRAIN)[0] == 0
    slot, planes = dec.decode(b)
    rc, got, _ = _apply(av1b, lib, torch, dec, b, slot)
    assert rc == 0
    for p in range(3):
        assert np.array_equal(got[p], planes[p])
    dec.release_reference(slot)


def _planted(av1b, payload, grain, restricted_identity):
    """A real stream's frame with the film grain block of `grain` planted (and,
    when asked, a restricted range clip with the identity colour matrix)."""
    raw = bytearray(payload)
    raw[_GRAIN:_GRAIN + _GRAIN_BYTES] = grain
    if restricted_identity:
        struct.pack_into('<i', raw, _CLIP, 1)
        struct.pack_into('<i', raw, _COLOR_MATRIX, 3)
    return av1b.Blob.from_bytes(bytes(raw))


@pytest.mark.parametrize('stream,restricted_identity', [
    ('lr_444', False),                  # 8-bit 4:4:4
    ('lr_422', False),                  # 8-bit 4:2:2
    ('aom_444_10bit_320x240', True),    # 10-bit 4:4:4, restricted range, identity matrix
    ('lr', True),                       # 8-bit 4:2:0, restricted range, identity matrix
])
def test_noalloc_subsampling_and_range_against_oracle(av1b, gpu, oracle, stream, restricted_identity):
    """The key frame of a real stream with film grain planted, decoded by the
    decoder and by the oracle; the entry point on the decoder's stored picture
    equals the oracle's output, sample for sample."""
    import stream_replay
    if stream not in stream_replay.fixture_names():
        pytest.skip('real-stream fixtures not built (make -C oracle streams)')
    dec, torch, lib = gpu
    fx = stream_replay.Fixture(stream)
    payload = fx.decodes()[0][3]
    donor = av1b.synth_frame(2, 8, 77, 0).to_bytes()
    grain = donor[_GRAIN:_GRAIN + _GRAIN_BYTES]
    assert struct.unpack_from('<i', grain, 0)[0] == 1
    b = _planted(av1b, payload, grain, restricted_identity)
    assert all(r < 0 for r in b.get_refs())   # a key frame: no references
    slot, mine = dec.decode(b)
    # the frame decoded last reads as its output picture (after grain); a
    # second decode makes `slot` an older slot, which reads as its stored
    # picture (before grain)
    again, _ = dec.decode(b)
    _, want = oracle.RefDecoder().decode(b)
    for p in range(3):
        assert np.array_equal(mine[p], want[p]), '%s decoder plane %d' % (stream, p)
    for n in range(2):  # two calls in a row
        rc, got, _ = _apply(av1b, lib, torch, dec, b, slot)
        assert rc == 0
        for p in range(3):
            assert np.array_equal(got[p], want[p]), '%s call %d plane %d' % (stream, n, p)
    dec.release_reference(slot)
    dec.release_reference(again)
