"""The oracle (TEST INFRASTRUCTURE ONLY; used by tests/, the smoke check and
bench.py's CPU-baseline leg and reference arm): the reference's own CPU
backend (built by oracle/Makefile into oracle/_ref/libav1ref.so) behind a
small Python class that mirrors av1ongpu_b200.Decoder.

Decoding through it loads libav1ref.so and nothing of this repository's
product: the plane and NV12 sizes are computed here, and a frame is any object
with the serialized blob's `ptr`, `size`, `header`, `get_refs` and `set_refs`
(RefBlob below, or av1ongpu_b200.Blob). Only `corrupt`, a fixture helper,
imports the product package, for its Blob type."""
import ctypes
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, 'oracle', '_ref', 'libav1ref.so')

_ref = None


def plane_shapes(width, height, ss_x, ss_y):
    """(rows, columns) of the three planes (Frame::plane_width / height)."""
    cw, ch = (width + ss_x) >> ss_x, (height + ss_y) >> ss_y
    return [(height, width), (ch, cw), (ch, cw)]


def nv12_size(width, height, ss_x, ss_y, pitch):
    """nv12_buffer_size (factory.cpp:236-244 of the reference): 4:2:0 only,
    an even pitch at least a chroma row wide; 0 otherwise."""
    if width <= 0 or height <= 0 or ss_x != 1 or ss_y != 1:
        return 0
    crow = 2 * ((width + 1) // 2)
    if pitch & 1 or pitch < crow:
        return 0
    return pitch * (height + (height + 1) // 2)


class RefBlob:
    """A serialized frame in a 64-byte aligned numpy buffer (the blob layout of
    av1ongpu_b200/csrc/flat_syntax.hpp: u32 magic, version, reserved, count,
    eight int32 reference slots, then the scalars from byte 48)."""

    def __init__(self, data):
        self._arr = np.zeros(len(data) + 64, dtype=np.uint8)
        off = (-self._arr.ctypes.data) % 64
        self._view = self._arr[off:off + len(data)]
        self._view[:] = np.frombuffer(data, dtype=np.uint8)
        self.ptr = self._view.ctypes.data
        self.size = len(data)

    @property
    def header(self):
        return struct.unpack_from('<6i', self._view, 48)

    def get_refs(self):
        n = struct.unpack_from('<I', self._view, 12)[0]
        return list(struct.unpack_from('<%di' % n, self._view, 16))

    def set_refs(self, slots):
        struct.pack_into('<I', self._view, 12, len(slots))
        struct.pack_into('<8i', self._view, 16, *(list(slots) + [-1] * (8 - len(slots))))


def available():
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_LIB)
        L.av1ref_create.restype = ctypes.c_void_p
        L.av1ref_destroy.argtypes = [ctypes.c_void_p]
        L.av1ref_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_size_t]
        L.av1ref_error.argtypes = [ctypes.c_void_p]
        L.av1ref_error.restype = ctypes.c_char_p
        L.av1ref_release.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.av1ref_to_nv12.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                     ctypes.c_size_t]
        L.av1ref_to_rgb.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_size_t]
        L.av1ref_set_threads.argtypes = [ctypes.c_int]
        L.av1ref_max_threads.restype = ctypes.c_int
        L.av1ref_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int)]
        L.av1ref_itx.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_void_p]
        L.av1ref_fnv1a64.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t]
        L.av1ref_fnv1a64.restype = ctypes.c_uint64
        L.av1ref_blob_counts.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        L.av1ref_dequant_pair.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32] + \
            [ctypes.c_void_p] * 4
        L.av1ref_free.argtypes = [ctypes.c_void_p]
        L.av1ref_strip.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p]
        L.av1ref_corrupt.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                                     ctypes.c_void_p, ctypes.c_void_p]
        _ref = L
    return _ref


class RefDecoder:
    def __init__(self):
        self.h = ref_lib().av1ref_create()
        if not self.h:
            raise RuntimeError('oracle decoder creation failed')

    def __del__(self):
        if getattr(self, 'h', None):
            ref_lib().av1ref_destroy(self.h)
            self.h = None

    def decode(self, blob, keep=True, read_back=True):
        w, _cw, h, _bd, sx, sy = blob.header
        shapes = plane_shapes(w, h, sx, sy)
        total = sum(a * b for a, b in shapes)
        out = np.empty(total, dtype=np.uint16) if read_back else None
        slot = ref_lib().av1ref_decode(self.h, blob.ptr, blob.size, 1 if keep else 0,
                                       out.ctypes.data if out is not None else None,
                                       total if out is not None else 0)
        if slot < -1:
            raise RuntimeError('oracle decode failed: %s' % ref_lib().av1ref_error(self.h).decode())
        planes = None
        if out is not None:
            planes, pos = [], 0
            for s in shapes:
                n = s[0] * s[1]
                planes.append(out[pos:pos + n].reshape(s))
                pos += n
        return slot, planes

    def release_reference(self, slot):
        ref_lib().av1ref_release(self.h, slot)

    def to_nv12(self, slot, pitch, width, height):
        n = nv12_size(width, height, 1, 1, pitch)
        out = np.empty(max(n, 1), dtype=np.uint8)
        got = ref_lib().av1ref_to_nv12(self.h, slot, pitch, out.ctypes.data, out.size)
        if got < 0:
            raise RuntimeError('oracle to_nv12 failed: %s' % ref_lib().av1ref_error(self.h).decode())
        return out[:got]

    def to_rgb(self, slot, matrix, rng, width, height):
        out = np.empty(width * height * 3, dtype=np.uint8)
        got = ref_lib().av1ref_to_rgb(self.h, slot, matrix, rng, out.ctypes.data, out.size)
        if got < 0:
            raise RuntimeError('oracle to_rgb failed')
        return out[:got]


def fnv1a64(arr, h=0xcbf29ce484222325):
    """FNV-1a 64 over the bytes of an array (the hash the reference's stream
    tests use, av1gpu_decode.cpp:131-140); `h` chains a previous result."""
    data = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    return ref_lib().av1ref_fnv1a64(h, data.ctypes.data, data.size)


BLOB_ARRAYS = ('blocks', 'transforms', 'obmc', 'coefficients', 'residual', 'levels', 'qm_pool',
               'palette_map', 'deblock', 'cdef', 'restoration')


def blob_counts(blob):
    """{array name: length} of a serialized frame (an av1ongpu_b200.Blob)."""
    out = (ctypes.c_uint64 * 11)()
    if ref_lib().av1ref_blob_counts(blob.ptr, blob.size, out) != 11:
        raise ValueError('malformed blob')
    return dict(zip(BLOB_ARRAYS, list(out)))


def dequant_pair(blob_bytes, seed):
    """(levels frame with seeded quantiser matrices, the same frame expanded
    into coefficient rasters by the reference front end's host dequantiser),
    both as serialized bytes, from a serialized levels frame."""
    src = RefBlob(blob_bytes)
    pa, pb = ctypes.c_void_p(), ctypes.c_void_p()
    na, nb = ctypes.c_size_t(), ctypes.c_size_t()
    L = ref_lib()
    if L.av1ref_dequant_pair(src.ptr, src.size, seed, ctypes.byref(pa), ctypes.byref(na),
                             ctypes.byref(pb), ctypes.byref(nb)):
        raise ValueError('malformed blob')
    try:
        return ctypes.string_at(pa, na.value), ctypes.string_at(pb, nb.value)
    finally:
        L.av1ref_free(pa)
        L.av1ref_free(pb)


DROP_DEBLOCK, DROP_CDEF, DROP_LR, DROP_GRAIN = 1, 2, 4, 8


def strip_stages(blob_bytes, drop):
    """A serialized frame without the in-loop stages named by `drop`
    (DROP_* bits), as bytes."""
    src = RefBlob(blob_bytes)
    p, n = ctypes.c_void_p(), ctypes.c_size_t()
    L = ref_lib()
    if L.av1ref_strip(src.ptr, src.size, drop, ctypes.byref(p), ctypes.byref(n)):
        raise ValueError('malformed blob')
    try:
        return ctypes.string_at(p, n.value)
    finally:
        L.av1ref_free(p)


CORRUPT_EDGE_LEVEL, CORRUPT_EDGE_OUTSIDE, CORRUPT_CDEF_DIR, CORRUPT_LR_UNIT, CORRUPT_GRAIN = 1, 2, 3, 4, 5


def corrupt(blob, what, index=0):
    """A copy of a serialized frame (an av1ongpu_b200.Blob) with one record
    made invalid (CORRUPT_*), as a new Blob."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import av1ongpu_b200 as av1b
    p, n = ctypes.c_void_p(), ctypes.c_size_t()
    L = ref_lib()
    if L.av1ref_corrupt(blob.ptr, blob.size, what, index, ctypes.byref(p), ctypes.byref(n)):
        raise ValueError('malformed blob or index')
    try:
        return av1b.Blob.from_bytes(ctypes.string_at(p, n.value))
    finally:
        L.av1ref_free(p)


def picture_hash(planes, bit_depth, yuv16):
    """The stream tests' frame hash of one picture: its planes in order, each
    sample one byte (shifted down to 8 bits) or two little endian bytes with
    `yuv16` (factory.cpp:194-233 of the reference)."""
    h = 0xcbf29ce484222325
    for p in planes:
        if yuv16:
            h = fnv1a64(np.ascontiguousarray(p, dtype='<u2'), h)
        else:
            h = fnv1a64((np.asarray(p) >> (bit_depth - 8)).astype(np.uint8), h)
    return h


class Stream:
    """Decodes a synthetic stream frame by frame with one decoder, mapping the
    generator's reference distances to that decoder's slots and releasing
    slots that no later frame can reference."""

    def __init__(self, dec, max_refs=3):
        self.dec = dec
        self.slots = {}
        self.max_refs = max_refs

    def decode(self, index, blob, keep=True, read_back=True):
        dists = blob.get_refs()
        blob.set_refs([self.slots[index - d] for d in dists])
        slot, planes = self.dec.decode(blob, keep=keep, read_back=read_back)
        blob.set_refs(dists)
        if keep:
            self.slots[index] = slot
        for k in [k for k in self.slots if k <= index - self.max_refs]:
            self.dec.release_reference(self.slots.pop(k))
        return slot, planes
