"""Writes a synthetic workload to files: one serialized FrameSyntax per frame.

    python -m av1ongpu_b200.workload --config 3 --seed 20261203 --frames 30 --out DIR

Frames come from the seeded generator (libav1synth.so) and are written as
DIR/frame_NNNN.av1s, their reference slot lists holding frame distances (1 =
the previous frame). A process that decodes them with another decoder - the
reference's CPU backend timed beside this library - then needs neither this
package's libraries nor the generator: only the bytes. The generator runs on
all host cores (each frame is independent of the others).
"""
import argparse
import os
import sys
from concurrent.futures import ThreadPoolExecutor


def write(config, scale, seed, frames, out):
    from . import synth_frame
    os.makedirs(out, exist_ok=True)

    def one(k):
        b = synth_frame(config, scale, seed, k)
        with open(os.path.join(out, 'frame_%04d.av1s' % k), 'wb') as f:
            f.write(b.to_bytes())
        return b.header

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        headers = list(ex.map(one, range(frames)))
    return headers[0]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--config', type=int, default=3)
    ap.add_argument('--scale', type=int, default=1)
    ap.add_argument('--seed', type=int, required=True)
    ap.add_argument('--frames', type=int, required=True)
    ap.add_argument('--out', required=True)
    args = ap.parse_args(argv)
    w, cw, h, bd, sx, sy = write(args.config, args.scale, args.seed, args.frames, args.out)
    print('%d %d %d %d %d %d' % (w, cw, h, bd, sx, sy))
    return 0


if __name__ == '__main__':
    sys.exit(main())
