"""Replays the real-stream fixtures (oracle/_ref/streams/*.av1s.gz, written by
oracle/stream_dump from the reference's 24 bit-exact test streams) through a
decoder that mirrors av1gpu::Decoder: decode_reference and release_reference
in the recorded order, show_existing_frame re-emitting an earlier picture,
and the frame hash of every shown picture compared with the stream's hash
list (the reference's stream tests, CMakeLists.txt:272-350 of the reference;
tools/av1gpu_decode.cpp:506-518 and 681-785 give the call order)."""
import gzip
import os
import struct

import av1ongpu_b200 as av1b
import refdec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STREAM_DIR = os.path.join(ROOT, 'oracle', '_ref', 'streams')

DECODE, RELEASE, SHOW_EXISTING = 1, 2, 3


def fixture_names(levels=False):
    if not os.path.isdir(STREAM_DIR):
        return []
    tail = '.levels.av1s.gz' if levels else '.av1s.gz'
    out = []
    for f in sorted(os.listdir(STREAM_DIR)):
        if f.endswith(tail) and (levels or not f.endswith('.levels.av1s.gz')):
            out.append(f[:-len(tail)])
    return out


class Fixture:
    def __init__(self, name, levels=False):
        path = os.path.join(STREAM_DIR, name + ('.levels' if levels else '') + '.av1s.gz')
        with gzip.open(path, 'rb') as f:
            data = f.read()
        magic, version, flags, n_hashes, n_events = struct.unpack_from('<4sIIII', data, 0)
        if magic != b'AV1S' or version != 1:
            raise ValueError('%s: not a replay fixture' % path)
        self.name = name
        self.yuv16 = bool(flags & 1)
        self.hashes = list(struct.unpack_from('<%dQ' % n_hashes, data, 32))
        pos = 32 + 8 * n_hashes
        self.events = []
        for _ in range(n_events):
            kind, a, b, _r, n = struct.unpack_from('<IiiIQ', data, pos)
            pos += 24
            self.events.append((kind, a, b, data[pos:pos + n]))
            pos += n
        if pos != len(data):
            raise ValueError('%s: %d trailing bytes' % (path, len(data) - pos))

    def decodes(self):
        return [e for e in self.events if e[0] == DECODE]


def replay(fx, dec, limit=None, keep_pictures=False, rewrite=None):
    """Runs the fixture's calls on `dec` (av1ongpu_b200.Decoder or
    refdec.RefDecoder). Returns (hashes of the shown pictures, pictures in
    decode order when keep_pictures else None). Slots are the decoder's own:
    the recorded ones are mapped as they are returned. `rewrite(k, bytes)`,
    when given, replaces the k-th decode's serialized frame."""
    slot_of = {-1: -1}
    shown_hash = []
    by_decode = []
    pictures = [] if keep_pictures else None
    for kind, a, b, payload in fx.events:
        if limit is not None and len(shown_hash) >= limit:
            break
        if kind == DECODE:
            if rewrite is not None:
                payload = rewrite(len(by_decode), payload)
            blob = av1b.Blob.from_bytes(payload)
            blob.set_refs([slot_of[s] for s in blob.get_refs()])
            bit_depth = blob.header[3]
            slot, planes = dec.decode(blob, keep=True, read_back=True)
            slot_of[a] = slot
            h = refdec.picture_hash(planes, bit_depth, fx.yuv16)
            by_decode.append(h)
            if keep_pictures:
                pictures.append(planes)
            if b:
                shown_hash.append(h)
        elif kind == RELEASE:
            dec.release_reference(slot_of.pop(a))
        elif kind == SHOW_EXISTING:
            shown_hash.append(by_decode[a])
        else:
            raise ValueError('unknown event %d' % kind)
    for s in [s for s in slot_of.values() if s >= 0]:
        dec.release_reference(s)
    return shown_hash, pictures
