"""A short decode for kernel profiles: the first frames of a synthetic
workload through the C ABI (plan, decode into reserved slots), nothing else.

    python -m av1ongpu_b200.profile_case --config 3 --scale 1 --frames 4

Frame 0 is the key frame (its dependency-scheduled phase is the longest);
frames 1.. are inter frames. Meant to run under a profiler with a kernel
filter and a launch count, e.g.
    ncu --set full --clock-control none -k regex:k_inter -s 1 -c 1 \\
        python -m av1ongpu_b200.profile_case
"""
import argparse
import ctypes
import sys

from . import Av1bError, Decoder, lib, synth_frame


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--config', type=int, default=3, help='workload (1..3)')
    ap.add_argument('--scale', type=int, default=1, help='divides the picture size')
    ap.add_argument('--frames', type=int, default=4)
    ap.add_argument('--seed', type=int, default=7)
    args = ap.parse_args(argv)
    dec = Decoder(0)
    ring = [dec.reserve_reference() for _ in range(4)]
    for k in range(args.frames):
        b = synth_frame(args.config, args.scale, args.seed, k)
        dists = b.get_refs()
        b.set_refs([ring[(k - d) % 4] for d in dists])
        view = ctypes.create_string_buffer(4096)
        if lib().av1b_syntax_view(b.ptr, b.size, view):
            raise Av1bError(-1, 'malformed frame')
        err = ctypes.create_string_buffer(256)
        rc = lib().av1b_decode_reserved(dec.h, view, ring[k % 4], None, err, 256)
        if rc:
            raise Av1bError(rc, err.value.decode())
    dec.close()
    print('decoded %d frames' % args.frames)
    return 0


if __name__ == '__main__':
    sys.exit(main())
