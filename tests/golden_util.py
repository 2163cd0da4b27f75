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


# The benchmark workloads at full size: name, (config, seed, frames, NV12
# pitch). bench_config3 is exactly the GOP bench.py times (its SEED, 30
# frames: 1 key + 29 inter); config 1 and 2 are the first 30 and 60 frames of
# their streams (seed 1000 * config), config 2 with its key frames at 0 and 30.
WORKLOADS = [
    ('bench_config3', (3, 20261203, 30, 4096)),
    ('config1_full', (1, 1000, 30, 1280)),
    ('config2_full', (2, 2000, 60, 1920)),
]
WORKLOAD_GOLDEN = os.path.join(HERE, 'golden', 'workloads.json')


def run_workload(dec, spec, av1b, frames=None):
    """Decodes a full-size workload with `dec` frame by frame; returns per
    frame [digest of the output planes, digest of the NV12 pack]."""
    import refdec
    config, seed, n, pitch = spec
    stream = refdec.Stream(dec)
    out = []
    for k in range(n if frames is None else frames):
        b = av1b.synth_frame(config, 1, seed, k)
        w, _, h, _, _, _ = b.header
        slot, planes = stream.decode(k, b)
        out.append([digest(planes), digest([dec.to_nv12(slot, pitch, w, h)])])
    for s in list(stream.slots.values()):
        dec.release_reference(s)
    return out


def load_workloads():
    with open(WORKLOAD_GOLDEN) as f:
        return json.load(f)['workloads']
