"""av1ongpu_b200: the B200 AV1 reconstruction backend, from Python.

A thin ctypes layer over the C ABI of libav1b.so (include/av1b.h). It mirrors
the reference library's av1gpu::Decoder (include/av1gpu/av1gpu.hpp:615-787 of
trprkkk/AV1onGPU): decode / decode_reference with device-resident reference
slots, release_reference, to_nv12, to_rgb and stats. Frames are passed as
serialized FrameSyntax blobs (`Blob`), which the seeded workload generator
(`synth_frame`, libav1synth.so, include/av1b_synth.h) produces. Importing the
package loads neither library; each is loaded at its first use.

There is no CPU path: without the compiled library, or without a CUDA device,
the calls raise instead of computing anything elsewhere.
"""
import ctypes
import os
import struct

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libav1b.so')
SYNTH_LIB_PATH = os.path.join(_HERE, 'libav1synth.so')

AV1B_OK = 0
ERRORS = {
    -1: 'bad argument', -2: 'CUDA error', -3: 'out of memory or slots', -4: 'invalid syntax',
    -5: 'device dependency wait timed out', -6: 'unsupported', -7: 'no CUDA device',
}

# workload tool bits (csrc/synth.cpp)
TOOL_TX64, TOOL_ALLTYPES, TOOL_CFL, TOOL_PALETTE = 1, 2, 4, 8
TOOL_FILTER_INTRA, TOOL_COMPOUND, TOOL_MASKS, TOOL_OBMC = 16, 32, 64, 128
TOOL_WARP, TOOL_LR, TOOL_GRAIN, TOOL_INTERINTRA = 256, 512, 1024, 2048
TOOL_INTRABC, TOOL_LOSSLESS, TOOL_RESIDUAL, TOOL_EDGE_VARIANTS = 4096, 8192, 16384, 32768
TOOL_NO_DEBLOCK, TOOL_NO_CDEF = 1 << 16, 1 << 17
TOOLS_ALL = (TOOL_TX64 | TOOL_ALLTYPES | TOOL_CFL | TOOL_PALETTE | TOOL_FILTER_INTRA |
             TOOL_COMPOUND | TOOL_MASKS | TOOL_OBMC | TOOL_WARP | TOOL_LR | TOOL_GRAIN |
             TOOL_EDGE_VARIANTS)


class Av1bError(RuntimeError):
    def __init__(self, code, msg=''):
        super().__init__('%s (%d)%s' % (ERRORS.get(code, 'error'), code, ': ' + msg if msg else ''))
        self.code = code


class _Planes(ctypes.Structure):
    _fields_ = [('plane', ctypes.c_void_p * 3), ('stride', ctypes.c_int32 * 3)]


class PlanInfo(ctypes.Structure):
    """av1b_plan_info: a planned frame's geometry and work counts."""
    _fields_ = [('width', ctypes.c_int32), ('height', ctypes.c_int32),
                ('coded_width', ctypes.c_int32), ('bit_depth', ctypes.c_int32),
                ('blocks', ctypes.c_int64), ('phase_b_blocks', ctypes.c_int64),
                ('chains', ctypes.c_int64), ('phase_b_samples', ctypes.c_int64),
                ('inter_tiles', ctypes.c_int64), ('inter_samples', ctypes.c_int64),
                ('inter_ref_samples', ctypes.c_int64), ('transforms', ctypes.c_int64),
                ('tx_samples', ctypes.c_int64), ('coef_samples', ctypes.c_int64),
                ('deblock_edges', ctypes.c_int64 * 2), ('cdef_blocks', ctypes.c_int64),
                ('lr_units', ctypes.c_int64), ('depth', ctypes.c_int32),
                ('upscaled', ctypes.c_int32), ('restored', ctypes.c_int32),
                ('grain', ctypes.c_int32)]

    def as_dict(self):
        out = {}
        for name, _t in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name == 'deblock_edges' else v
        return out


class BatchConfig(ctypes.Structure):
    """av1b_batch_config: the batched step's launch shape."""
    _fields_ = [('ctas_per_sm', ctypes.c_int32 * 24), ('claim_chunk', ctypes.c_int32),
                ('fuse_grain_nv12', ctypes.c_int32), ('use_graph', ctypes.c_int32),
                ('inter_variant', ctypes.c_int32)]

    def as_dict(self):
        return {'ctas_per_sm': list(self.ctas_per_sm)[:len(Batch.STAGES)], 'claim_chunk': self.claim_chunk,
                'fuse_grain_nv12': self.fuse_grain_nv12, 'use_graph': self.use_graph,
                'inter_variant': self.inter_variant}


class ServerResult(ctypes.Structure):
    """av1b_server_result: one completed frame of the served form."""
    _fields_ = [('stream_id', ctypes.c_int32), ('status', ctypes.c_int32), ('slot', ctypes.c_int32),
                ('batch_size', ctypes.c_int32), ('tag', ctypes.c_uint64),
                ('frame_index', ctypes.c_uint64), ('step', ctypes.c_int64),
                ('arrival_ms', ctypes.c_double), ('done_ms', ctypes.c_double),
                ('latency_ms', ctypes.c_double), ('planned_ms', ctypes.c_double),
                ('nv12_device', ctypes.c_void_p),
                ('nv12_bytes', ctypes.c_size_t)]


class ServerStats(ctypes.Structure):
    _fields_ = [('submitted', ctypes.c_uint64), ('completed', ctypes.c_uint64),
                ('steps', ctypes.c_uint64), ('stepped_frames', ctypes.c_uint64),
                ('hbm_used', ctypes.c_size_t), ('hbm_budget', ctypes.c_size_t),
                ('streams', ctypes.c_int32), ('now_ms', ctypes.c_double),
                ('plan_ms', ctypes.c_double), ('launch_ms', ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [('blocks', ctypes.c_int32), ('waves', ctypes.c_int32),
                ('kernel_launches', ctypes.c_int32), ('reconstruct_ms', ctypes.c_double),
                ('filter_ms', ctypes.c_double), ('readback_ms', ctypes.c_double),
                ('total_ms', ctypes.c_double)]


_lib = None

# name: (restype, argtypes)
_SIGNATURES = {
    'av1b_syntax_view': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    'av1b_decoder_create': (ctypes.c_int, [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    'av1b_decoder_create_ex': (ctypes.c_int, [ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_void_p)]),
    'av1b_decoder_destroy': (ctypes.c_int, [ctypes.c_void_p]),
    'av1b_decoder_reset': (ctypes.c_int, [ctypes.c_void_p]),
    'av1b_decode': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_size_t]),
    'av1b_decode_blob': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                        ctypes.c_size_t]),
    'av1b_reserve_reference': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    'av1b_plan_frame': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    'av1b_decode_planned': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    'av1b_plan_free': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    'av1b_sync': (ctypes.c_int, [ctypes.c_void_p]),
    'av1b_plan_stats': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    'av1b_batch_create': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    'av1b_batch_destroy': (ctypes.c_int, [ctypes.c_void_p]),
    'av1b_batch_decode': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    'av1b_batch_sync': (ctypes.c_int, [ctypes.c_void_p]),
    'av1b_batch_get_config': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    'av1b_batch_set_config': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    'av1b_batch_autotune': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    'av1b_batch_last_error': (ctypes.c_char_p, [ctypes.c_void_p]),
    'av1b_batch_set_profiling': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_batch_profile': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_longlong)]),
    'av1b_server_create': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    'av1b_server_destroy': (ctypes.c_int, [ctypes.c_void_p]),
    'av1b_server_open': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_size_t)]),
    'av1b_server_close': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_server_submit': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                          ctypes.c_uint64]),
    'av1b_server_poll': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int)]),
    'av1b_server_drain': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_server_get_stats': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    'av1b_server_batch': (ctypes.c_void_p, [ctypes.c_void_p]),
    'av1b_stream_hbm_estimate': (ctypes.c_size_t, [ctypes.c_int] * 8),
    'av1b_decoder_memory': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                           ctypes.POINTER(ctypes.c_size_t)]),
    'av1b_batch_stream': (ctypes.c_void_p, [ctypes.c_void_p]),
    'av1b_int_peak': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    'av1b_handoff_peak': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    'av1b_set_shared_masks': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_set_profiling': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_set_wait_limit': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    'av1b_selftest_wait': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double)]),
    'av1b_profile': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]),
    'av1b_decode_reserved': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    'av1b_release_reference': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_to_nv12': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                    ctypes.c_size_t]),
    'av1b_to_nv12_device': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t,
                                           ctypes.c_void_p, ctypes.c_size_t]),
    'av1b_nv12_size': (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_size_t]),
    'av1b_nv12_pack_begin': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_int)]),
    'av1b_nv12_pack_wait': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_size_t, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_size_t)]),
    'av1b_nv12_pack_release': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_to_rgb': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_size_t]),
    'av1b_get_stats': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Stats)]),
    'av1b_poll_status': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    'av1b_slot_planes_device': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_void_p]),
    'av1b_last_error': (ctypes.c_char_p, [ctypes.c_void_p]),
    'av1b_set_unit_trace': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'av1b_unit_trace': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t)]),
    'av1b_decoder_stream': (ctypes.c_void_p, [ctypes.c_void_p]),
    'av1b_blob_set_refs': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.c_int]),
    'av1b_blob_get_refs': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.c_int]),
}


_SYNTH_SIGNATURES = {
    'av1s_synth_frame': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]),
    'av1s_synth_frame_ex': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_size_t)]),
    'av1s_synth_frame_refs': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                             ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                             ctypes.POINTER(ctypes.c_size_t)]),
    'av1s_blob_free': (None, [ctypes.c_void_p]),
}
_synth = None


def synth_lib():
    """Loads libav1synth.so, the workload generator (raises if it was not built)."""
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_LIB_PATH):
            raise OSError('libav1synth.so is not built: run python -m av1ongpu_b200.build')
        L = ctypes.CDLL(SYNTH_LIB_PATH)
        for name, (res, args) in _SYNTH_SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _synth = L
    return _synth


def lib():
    """Loads libav1b.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError('libav1b.so is not built: run python -m av1ongpu_b200.build')
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def synth_exported_symbols():
    return list(_SYNTH_SIGNATURES)


# ---- serialized frames -----------------------------------------------------------------------
_BLOB_HEADER = 48  # magic, version, reserved, n_refs, ref_slots[8]
_BLOB_MAGIC = 0x42315641  # "AV1B"


class Blob:
    """A serialized FrameSyntax, 64-byte aligned, owned by the generator library
    or by numpy. The header (geometry and the patchable reference slot list)
    is read and written here directly, without either library."""

    def __init__(self, ptr, size, owned_by_lib):
        self.ptr = ptr
        self.size = size
        self._lib_owned = owned_by_lib
        self._keep = None

    @classmethod
    def from_bytes(cls, data):
        arr = np.zeros(len(data) + 64, dtype=np.uint8)
        off = (-arr.ctypes.data) % 64
        view = arr[off:off + len(data)]
        view[:] = np.frombuffer(data, dtype=np.uint8)
        b = cls(view.ctypes.data, len(data), False)
        b._keep = arr
        return b

    def to_bytes(self):
        return ctypes.string_at(self.ptr, self.size)

    def __del__(self):
        if self._lib_owned and self.ptr and _synth is not None:
            _synth.av1s_blob_free(ctypes.c_void_p(self.ptr))
            self.ptr = None

    def _head(self):
        if self.size < _BLOB_HEADER:
            raise Av1bError(-1, 'malformed blob')
        magic, _version, _r, n = struct.unpack_from('<4I', ctypes.string_at(self.ptr, 16))
        if magic != _BLOB_MAGIC or n > 8:
            raise Av1bError(-1, 'malformed blob')
        return n

    @property
    def header(self):
        """(width, coded_width, height, bit_depth, ss_x, ss_y)."""
        return struct.unpack_from('<6i', ctypes.string_at(self.ptr + _BLOB_HEADER, 24))

    def get_refs(self):
        n = self._head()
        return list(struct.unpack_from('<%di' % n, ctypes.string_at(self.ptr + 16, 4 * n)))

    def set_refs(self, slots):
        self._head()
        if len(slots) > 8:
            raise Av1bError(-1, 'more than eight reference slots')
        ctypes.memmove(self.ptr + 12, struct.pack('<I', len(slots)), 4)
        vals = list(slots) + [-1] * (8 - len(slots))
        ctypes.memmove(self.ptr + 16, struct.pack('<8i', *vals), 32)


def synth_frame(config, scale, seed, index):
    """One frame of workload `config` (1..3) at 1/scale size."""
    p = ctypes.c_void_p()
    n = ctypes.c_size_t()
    rc = synth_lib().av1s_synth_frame(config, scale, seed, index, ctypes.byref(p), ctypes.byref(n))
    if rc:
        raise Av1bError(rc, 'synth_frame')
    return Blob(p.value, n.value, True)


def synth_frame_ex(width, height, coded_width, bit_depth, sb_size, tools, seed, index,
                   key_interval=0, max_refs=None):
    """A frame of any geometry (tools: the TOOL_* bits); `max_refs` the
    reference slots an inter frame draws from (default: 3 with compound
    prediction, else 1)."""
    p = ctypes.c_void_p()
    n = ctypes.c_size_t()
    if max_refs is None:
        rc = synth_lib().av1s_synth_frame_ex(width, height, coded_width, bit_depth, sb_size, tools,
                                             seed, index, key_interval, ctypes.byref(p),
                                             ctypes.byref(n))
    else:
        rc = synth_lib().av1s_synth_frame_refs(width, height, coded_width, bit_depth, sb_size,
                                               tools, max_refs, seed, index, key_interval,
                                               ctypes.byref(p), ctypes.byref(n))
    if rc:
        raise Av1bError(rc, 'synth_frame_ex')
    return Blob(p.value, n.value, True)


def plane_shapes(width, height, ss_x, ss_y):
    cw, ch = (width + ss_x) >> ss_x, (height + ss_y) >> ss_y
    return [(height, width), (ch, cw), (ch, cw)]


def nv12_size(width, height, ss_x, ss_y, pitch):
    return lib().av1b_nv12_size(width, height, ss_x, ss_y, pitch)


# ---- the decoder -----------------------------------------------------------------------------
class Decoder:
    """av1gpu::Decoder on one CUDA device."""

    def __init__(self, device=0, hbm_budget=0, planners=0, planner_threads=0):
        h = ctypes.c_void_p()
        opt = (ctypes.c_int32 * 2)(planners, planner_threads)
        rc = lib().av1b_decoder_create_ex(device, hbm_budget, opt, ctypes.byref(h))
        if rc:
            raise Av1bError(rc, 'av1b_decoder_create')
        self.h = h
        self._err = ctypes.create_string_buffer(512)

    def close(self):
        if getattr(self, 'h', None):
            lib().av1b_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = lib().av1b_last_error(self.h) or b''
            raise Av1bError(rc, '%s: %s' % (what, msg.decode(errors='replace')))

    def decode(self, blob, keep=True, read_back=True):
        """Decodes a serialized frame. Returns (slot, [Y, U, V] uint16 arrays or None)."""
        w, _cw, h, _bd, sx, sy = blob.header
        planes = None
        pl = None
        if read_back:
            planes = [np.empty(s, dtype=np.uint16) for s in plane_shapes(w, h, sx, sy)]
            pl = _Planes()
            for i, a in enumerate(planes):
                pl.plane[i] = a.ctypes.data
                pl.stride[i] = a.shape[1]
        slot = ctypes.c_int(-1)
        rc = lib().av1b_decode_blob(self.h, blob.ptr, blob.size, 1 if keep else 0,
                                    ctypes.byref(pl) if pl is not None else None, ctypes.byref(slot),
                                    self._err, len(self._err))
        self._check(rc, 'decode')
        return slot.value, planes

    def plan(self, blob):
        """Plans a serialized frame: validation and upload of its device records.
        Returns an opaque plan handle for decode_planned."""
        view = ctypes.create_string_buffer(4096)
        rc = lib().av1b_syntax_view(blob.ptr, blob.size, view)
        if rc:
            raise Av1bError(rc, 'malformed blob')
        h = ctypes.c_void_p()
        self._check(lib().av1b_plan_frame(self.h, view, ctypes.byref(h)), 'plan_frame')
        return h

    def decode_planned(self, plan, slot=-1, keep=True, wait=True, planes=None):
        pl = None
        if planes is not None:
            pl = _Planes()
            for i, a in enumerate(planes):
                pl.plane[i] = a.ctypes.data
                pl.stride[i] = a.shape[1]
        got = ctypes.c_int(-1)
        rc = lib().av1b_decode_planned(self.h, plan, slot, 1 if keep else 0,
                                       ctypes.byref(pl) if pl is not None else None,
                                       ctypes.byref(got), 1 if wait else 0)
        self._check(rc, 'decode_planned')
        return got.value

    def plan_stats(self, plan):
        """The planned frame's work counts (av1b_plan_stats) as a dict."""
        info = PlanInfo()
        self._check(lib().av1b_plan_stats(plan, ctypes.byref(info)), 'plan_stats')
        return info.as_dict()

    def free_plan(self, plan):
        self._check(lib().av1b_plan_free(self.h, plan), 'plan_free')

    def selftest_wait(self, limit_ns):
        st = ctypes.c_int(0)
        ms = ctypes.c_double(0)
        self._check(lib().av1b_selftest_wait(self.h, limit_ns, ctypes.byref(st), ctypes.byref(ms)),
                    'selftest_wait')
        return st.value, ms.value

    def set_wait_limit(self, limit_ns):
        self._check(lib().av1b_set_wait_limit(self.h, limit_ns), 'set_wait_limit')

    def set_profiling(self, on):
        self._check(lib().av1b_set_profiling(self.h, 1 if on else 0), 'set_profiling')

    def set_shared_masks(self, on):
        """Chroma blocks of difference-weighted compounds read their luma
        block's mask (on, the default) or predict the luma themselves (off):
        the same samples either way."""
        self._check(lib().av1b_set_shared_masks(self.h, 1 if on else 0), 'set_shared_masks')

    def set_unit_trace(self, on):
        self._check(lib().av1b_set_unit_trace(self.h, 1 if on else 0), 'set_unit_trace')

    def unit_trace(self):
        """The last frame's phase B trace: an (n_blocks, 4) uint64 array of
        (claimed, ready, published) globaltimer ns and the dependency
        published last, zero rows for blocks outside phase B."""
        n = ctypes.c_size_t(0)
        self._check(lib().av1b_unit_trace(self.h, None, 0, ctypes.byref(n)), 'unit_trace')
        out = np.zeros(n.value, dtype=np.uint64)
        if n.value:
            self._check(lib().av1b_unit_trace(self.h, out.ctypes.data, n.value, ctypes.byref(n)),
                        'unit_trace')
        return out.reshape(-1, 4)

    def profile(self):
        """{stage: (total_ms, launches)} since profiling was switched on."""
        out = {}
        i = 0
        while True:
            name = ctypes.c_char_p()
            ms = ctypes.c_double()
            n = ctypes.c_longlong()
            r = lib().av1b_profile(self.h, i, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(n))
            if r != 1:
                break
            out[name.value.decode()] = (ms.value, n.value)
            i += 1
        return out

    def sync(self):
        self._check(lib().av1b_sync(self.h), 'sync')

    def stream(self):
        return lib().av1b_decoder_stream(self.h)

    def to_nv12_device(self, slot, pitch, dst_ptr, dst_len):
        self._check(lib().av1b_to_nv12_device(self.h, slot, pitch, dst_ptr, dst_len), 'to_nv12_device')

    def reserve_reference(self):
        s = ctypes.c_int(-1)
        self._check(lib().av1b_reserve_reference(self.h, ctypes.byref(s)), 'reserve_reference')
        return s.value

    def release_reference(self, slot):
        self._check(lib().av1b_release_reference(self.h, slot), 'release_reference')

    def reset(self):
        self._check(lib().av1b_decoder_reset(self.h), 'reset')

    def to_nv12(self, slot, pitch, width, height):
        n = nv12_size(width, height, 1, 1, pitch)
        if n == 0:
            raise Av1bError(-1, 'NV12 needs a 4:2:0 frame and an even pitch at least as wide')
        out = np.empty(n, dtype=np.uint8)
        self._check(lib().av1b_to_nv12(self.h, slot, pitch, out.ctypes.data, n), 'to_nv12')
        return out

    def nv12_pack_begin(self, slot, pitch):
        """Starts packing `slot` as NV12 (device pack, read back on a side
        stream into page-locked memory); returns a handle for nv12_pack_wait."""
        h = ctypes.c_int(-1)
        self._check(lib().av1b_nv12_pack_begin(self.h, slot, pitch, ctypes.byref(h)),
                    'nv12_pack_begin')
        return h.value

    def nv12_pack_wait(self, handle, out=None):
        """Waits for a pack. With `out` (a uint8 array) the bytes are copied
        into it and it is returned; without, a uint8 view of the page-locked
        bytes is returned, valid until nv12_pack_release."""
        data = ctypes.c_void_p()
        n = ctypes.c_size_t(0)
        if out is not None:
            self._check(lib().av1b_nv12_pack_wait(self.h, handle, out.ctypes.data, out.nbytes, None,
                                                  ctypes.byref(n)), 'nv12_pack_wait')
            return out[:n.value]
        self._check(lib().av1b_nv12_pack_wait(self.h, handle, None, 0, ctypes.byref(data),
                                              ctypes.byref(n)), 'nv12_pack_wait')
        buf = (ctypes.c_uint8 * n.value).from_address(data.value)
        return np.frombuffer(buf, dtype=np.uint8)

    def nv12_pack_release(self, handle):
        self._check(lib().av1b_nv12_pack_release(self.h, handle), 'nv12_pack_release')

    def to_rgb(self, slot, matrix, rng, width, height):
        out = np.empty(width * height * 3, dtype=np.uint8)
        self._check(lib().av1b_to_rgb(self.h, slot, matrix, rng, out.ctypes.data, out.size), 'to_rgb')
        return out

    def stats(self):
        s = Stats()
        self._check(lib().av1b_get_stats(self.h, ctypes.byref(s)), 'stats')
        return s


class Batch:
    """The batched form (av1b_batch_*): one planned frame of each of many
    streams - each a Decoder of its own - decoded as one step of persistent
    kernels replayed as a CUDA graph."""

    MAX = 64

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = lib().av1b_batch_create(device, ctypes.byref(h))
        if rc:
            raise Av1bError(rc, 'av1b_batch_create')
        self.h = h

    def close(self):
        if getattr(self, 'h', None):
            lib().av1b_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = lib().av1b_batch_last_error(self.h) or b''
            raise Av1bError(rc, '%s: %s' % (what, msg.decode(errors='replace')))

    @staticmethod
    def _args(decoders, plans, slots, nv12):
        n = len(decoders)
        decs = (ctypes.c_void_p * n)(*[d.h.value for d in decoders])
        pls = (ctypes.c_void_p * n)(*[p.value for p in plans])
        sl = (ctypes.c_int * n)(*(slots if slots is not None else [-1] * n))
        dst = pitch = length = None
        if nv12 is not None:
            dst = (ctypes.c_void_p * n)(*[x[0] if x else None for x in nv12])
            pitch = (ctypes.c_size_t * n)(*[x[1] if x else 0 for x in nv12])
            length = (ctypes.c_size_t * n)(*[x[2] if x else 0 for x in nv12])
        return n, decs, pls, sl, dst, pitch, length

    def decode(self, decoders, plans, slots=None, nv12=None):
        """Queues one step: frame i = plans[i] on decoders[i] into slots[i]
        (-1: lowest free); nv12[i] = (device pointer, pitch, bytes) or None.
        Returns the slots."""
        n, decs, pls, sl, dst, pitch, length = self._args(decoders, plans, slots, nv12)
        out = (ctypes.c_int * n)()
        self._check(lib().av1b_batch_decode(self.h, n, decs, pls, sl, out, dst, pitch, length),
                    'batch_decode')
        return list(out)

    def sync(self):
        self._check(lib().av1b_batch_sync(self.h), 'batch_sync')

    def config(self):
        c = BatchConfig()
        self._check(lib().av1b_batch_get_config(self.h, ctypes.byref(c)), 'batch_get_config')
        return c

    def set_config(self, c):
        self._check(lib().av1b_batch_set_config(self.h, ctypes.byref(c)), 'batch_set_config')

    def autotune(self, decoders, plans, slots=None, nv12=None, cache_path=None, reps=3):
        """Picks the launch shape for this set of streams (see av1b.h);
        returns (config dict, best step ms or -1 when taken from the cache)."""
        n, decs, pls, sl, dst, pitch, length = self._args(decoders, plans, slots, nv12)
        c = BatchConfig()
        ms = ctypes.c_double(0)
        path = cache_path.encode() if cache_path else None
        self._check(lib().av1b_batch_autotune(self.h, n, decs, pls, sl, dst, pitch, length, path,
                                              reps, ctypes.byref(c), ctypes.byref(ms)),
                    'batch_autotune')
        return c.as_dict(), ms.value

    def stream(self):
        return lib().av1b_batch_stream(self.h)

    STAGES = ('inter_simple', 'inter_lean_mask', 'inter', 'inter_mask', 'itx4', 'itx8', 'itx16', 'itx32', 'itx64', 'itx_raw', 'units',
              'deblock_v', 'deblock_h', 'copy_snapshot', 'cdef_search', 'cdef', 'copy_post_cdef',
              'upscale', 'lr', 'copy_reference', 'grain_template', 'grain_blend', 'nv12')

    def set_profiling(self, on):
        self._check(lib().av1b_batch_set_profiling(self.h, 1 if on else 0), 'batch_set_profiling')

    def profile(self):
        """{stage: total ms} over the steps timed, and the step count."""
        out, n = {}, 0
        for k, name in enumerate(self.STAGES):
            ms = ctypes.c_double(0)
            steps = ctypes.c_longlong(0)
            self._check(lib().av1b_batch_profile(self.h, k, ctypes.byref(ms), ctypes.byref(steps)),
                        'batch_profile')
            out[name] = ms.value
            n = steps.value
        return out, n


class Server:
    """The served form (av1b_server_*): streams admitted by HBM, frame
    requests planned as they arrive and run in continuously batched steps."""

    def __init__(self, device=0, max_batch=0, max_inflight=0, planner_threads=0, hbm_budget=0,
                 decoder_threads=0, batch_wait_us=0):
        opt = (ctypes.c_int32 * 6)(device, max_batch, max_inflight, planner_threads, decoder_threads,
                                   batch_wait_us)
        buf = ctypes.create_string_buffer(bytes(opt) + bytes(ctypes.c_size_t(hbm_budget)))
        h = ctypes.c_void_p()
        rc = lib().av1b_server_create(buf, ctypes.byref(h))
        if rc:
            raise Av1bError(rc, 'av1b_server_create')
        self.h = h

    def close(self):
        if getattr(self, 'h', None):
            lib().av1b_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def open(self, width, height, bit_depth, coded_width=0, ss_x=1, ss_y=1, max_refs=3,
             nv12_pitch=0):
        """Admits a stream; returns (stream id, HBM bytes reserved). Raises
        Av1bError(-3) when it does not fit the server's budget now."""
        desc = (ctypes.c_int32 * 8)(width, height, coded_width, bit_depth, ss_x, ss_y, max_refs,
                                    nv12_pitch)
        sid = ctypes.c_int(-1)
        hbm = ctypes.c_size_t(0)
        rc = lib().av1b_server_open(self.h, desc, ctypes.byref(sid), ctypes.byref(hbm))
        if rc:
            raise Av1bError(rc, 'server_open')
        return sid.value, hbm.value

    def close_stream(self, sid):
        rc = lib().av1b_server_close(self.h, sid)
        if rc:
            raise Av1bError(rc, 'server_close')

    def submit(self, sid, blob, tag=0):
        rc = lib().av1b_server_submit(self.h, sid, blob.ptr, blob.size, tag)
        if rc:
            raise Av1bError(rc, 'server_submit')

    def poll(self, max_results=256, wait_ms=0):
        out = (ServerResult * max_results)()
        n = ctypes.c_int(0)
        rc = lib().av1b_server_poll(self.h, out, max_results, wait_ms, ctypes.byref(n))
        if rc:
            raise Av1bError(rc, 'server_poll')
        return [out[i] for i in range(n.value)]

    def drain(self, timeout_ms=60000):
        rc = lib().av1b_server_drain(self.h, timeout_ms)
        if rc:
            raise Av1bError(rc, 'server_drain')

    def stats(self):
        st = ServerStats()
        rc = lib().av1b_server_get_stats(self.h, ctypes.byref(st))
        if rc:
            raise Av1bError(rc, 'server_stats')
        return st

    def batch_handle(self):
        return lib().av1b_server_batch(self.h)


def int_peak(device=0, kind=0):
    """32-bit operations per second the SMs issue (av1b_int_peak): independent
    adds (kind 0) or multiply-adds (kind 1)."""
    v = ctypes.c_double(0)
    rc = lib().av1b_int_peak(device, kind, ctypes.byref(v))
    if rc:
        raise Av1bError(rc, 'int_peak')
    return v.value


def handoff_peak(device=0):
    """The floor of a dependency step (av1b_handoff_peak): the median one-way
    ns of a flag handed between warps on two SMs by a release store and
    acquire polls."""
    v = ctypes.c_double(0)
    rc = lib().av1b_handoff_peak(device, ctypes.byref(v))
    if rc:
        raise Av1bError(rc, 'handoff_peak')
    return v.value


def cuda_available():
    """True when a CUDA device is visible (without initialising torch)."""
    try:
        rt = ctypes.CDLL('libcudart.so')
    except OSError:
        try:
            import glob
            cands = glob.glob('/usr/local/cuda/lib64/libcudart.so*')
            rt = ctypes.CDLL(cands[0]) if cands else None
        except OSError:
            rt = None
    if rt is None:
        return False
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
