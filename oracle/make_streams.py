"""Writes the real-stream replay fixtures (TEST INFRASTRUCTURE ONLY).

    python3 oracle/make_streams.py --ref REFERENCE_CHECKOUT \\
        --tool oracle/_ref/stream_dump --out oracle/_ref/streams

Runs stream_dump (oracle/stream_dump.cpp) over the reference's 24 bit-exact
test streams, with the frame counts and sample widths its stream tests use
(CMakeLists.txt:272-350 of the reference: `--frames`, and `--yuv16` for the
streams deeper than 8 bits). Each fixture is written twice: `NAME.av1s.gz`
with dequantised coefficients, and `NAME.levels.av1s.gz` planned for a device
dequantiser (coded levels, steps and QM offsets). stream_dump checks the
reference's own output against the stream's hash list before it writes
anything, so a fixture exists only for a stream the reference decodes bit
exactly."""
import argparse
import gzip
import os
import subprocess
import sys

# name: (frames, 16-bit hashes)
STREAMS = {
    'lw_t2': (30, False), 'lw_t3': (30, False), 'palette_sc': (10, False),
    'intrabc': (16, False), 'inter_intra': (110, False), 'seg_altq': (30, False),
    'superres': (30, False), 'grain': (30, False), 'grain_inherit': (10, False),
    'lr': (8, False), 'lr_10bit': (8, True), 'lr_12bit': (8, True),
    'lr_444': (8, False), 'lr_422': (8, False), 'lossless': (4, False),
    'odd_size': (6, False), 'edge_grid': (4, False), 'tiles': (4, False),
    'tiles_grid': (4, False), 'aom_10bit_320x240': (12, True),
    'aom_444_10bit_320x240': (12, True), 'aom_12bit_320x240': (12, True),
    'palette_10bit': (2, True), 'error_resilient': (4, False),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--ref', required=True, help='reference checkout (has tests/data)')
    ap.add_argument('--tool', required=True, help='the stream_dump binary')
    ap.add_argument('--out', required=True, help='output folder')
    ap.add_argument('--only', nargs='*', help='stream names (default: all)')
    args = ap.parse_args(argv)
    os.makedirs(args.out, exist_ok=True)
    data = os.path.join(args.ref, 'tests', 'data')
    failed = []
    for name in args.only or sorted(STREAMS):
        frames, deep = STREAMS[name]
        for suffix, extra in (('', []), ('.levels', ['--levels'])):
            raw = os.path.join(args.out, name + suffix + '.av1s')
            cmd = [args.tool, os.path.join(data, name + '.ivf'), '--frames', str(frames),
                   '--hashes', os.path.join(data, name + '.hash'), '-o', raw] + extra
            if deep:
                cmd.append('--yuv16')
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                failed.append(name + suffix)
                sys.stderr.write(r.stderr)
                continue
            with open(raw, 'rb') as f, gzip.open(raw + '.gz', 'wb', compresslevel=6) as g:
                g.write(f.read())
            os.remove(raw)
            print(r.stdout.strip())
    if failed:
        print('not written: %s' % ' '.join(failed), file=sys.stderr)
        return 1
    return 0


if __name__ == '__main__':
    sys.exit(main())
