"""Golden fixtures: per-frame hashes of the oracle's output on seeded
synthetic streams, committed in tests/golden/golden.json and regenerated by
tests/golden/make_golden.py. A GPU run without the oracle build still has
these to compare against."""
import hashlib
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, 'golden', 'golden.json')

# name, generator args (width, height, coded_width, bit_depth, sb, tools, key_interval), frames
TOOLS_ALL = 0xFFFF & ~(2048 | 4096 | 8192 | 16384)


def cases_spec(av1b):
    A = av1b
    return [
        ('c1_160x96', (160, 96, 0, 8, 64, 0, 0), 3),
        ('c1_odd_150x90', (150, 90, 0, 8, 64, 0, 0), 3),
        ('c2_240x136_all', (240, 136, 0, 10, 64, A.TOOLS_ALL, 30), 3),
        ('c3_480x270_superres', (480, 270, 360, 10, 128, A.TOOLS_ALL, 30), 3),
        ('extras_interintra_intrabc_residual', (240, 136, 0, 10, 64,
                                               A.TOOLS_ALL | A.TOOL_INTERINTRA | A.TOOL_INTRABC |
                                               A.TOOL_RESIDUAL, 30), 3),
        ('lossless_8bit', (160, 96, 0, 8, 64, A.TOOL_LOSSLESS, 0), 2),
        ('c2_12bit', (192, 128, 0, 12, 64, A.TOOLS_ALL, 30), 2),
    ]


def digest(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(a.tobytes())
    return h.hexdigest()[:32]


def run_case(dec, case, av1b, seed=4242):
    import refdec
    stream = refdec.Stream(dec)
    prm = case['params']
    out = []
    w, h = prm[0], prm[1]
    pitch = (w + 63) & ~63
    for k in range(case['n']):
        b = av1b.synth_frame_ex(*prm[:6], seed, k, prm[6])
        slot, planes = stream.decode(k, b)
        nv12 = dec.to_nv12(slot, pitch, w, h)
        out.append([digest(planes), digest([nv12])])
    return out


def load():
    with open(GOLDEN) as f:
        return json.load(f)['cases']
