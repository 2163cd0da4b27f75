"""Regenerates the golden fixtures from the oracle (the reference CPU backend
built by oracle/Makefile). Run in the build container:

    make -C oracle REF=<reference checkout> && python tests/golden/make_golden.py [--workloads]

golden.json: per-frame hashes of small seeded streams of every tool mix.
workloads.json (--workloads, a few minutes): per-frame hashes of the full-size
benchmark workloads (golden_util.WORKLOADS), which bench.py checks the frames
it times against before timing them.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, 'oracle'), os.path.dirname(HERE)]

import av1ongpu_b200 as av1b  # noqa: E402
import golden_util  # noqa: E402
import refdec  # noqa: E402


def make_workloads():
    refdec.ref_lib().av1ref_set_threads(os.cpu_count() or 1)
    out = {}
    for name, spec in golden_util.WORKLOADS:
        frames = golden_util.run_workload(refdec.RefDecoder(), spec, av1b)
        out[name] = {'config': spec[0], 'seed': spec[1], 'frames_n': spec[2], 'pitch': spec[3],
                     'frames': frames}
        print(name, len(frames), frames[-1])
    with open(golden_util.WORKLOAD_GOLDEN, 'w') as f:
        json.dump({'generator': 'tests/golden/make_golden.py --workloads', 'workloads': out}, f,
                  indent=1)


def main():
    if '--workloads' in sys.argv:
        make_workloads()
        return
    cases = []
    for name, params, n in golden_util.cases_spec(av1b):
        case = {'name': name, 'params': list(params), 'n': n}
        case['frames'] = golden_util.run_case(refdec.RefDecoder(), case, av1b)
        cases.append(case)
        print(name, case['frames'][-1])
    with open(golden_util.GOLDEN, 'w') as f:
        json.dump({'generator': 'tests/golden/make_golden.py', 'seed': 4242, 'cases': cases}, f,
                  indent=1)


if __name__ == '__main__':
    main()
