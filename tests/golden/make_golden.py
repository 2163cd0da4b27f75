"""Regenerates tests/golden/golden.json from the oracle (the reference CPU
backend built by oracle/Makefile). Run in the build container:

    make -C oracle && python tests/golden/make_golden.py
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


def main():
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
