"""bench.py's reference arm on the CPU: it times the reference's CPU backend
on the same GOP and configuration as the GPU arm, and its process maps the
reference's library only - the workload is written by a separate process, so
neither this repository's decoder nor its generator is loaded."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r'''
import sys
sys.argv = ['bench.py', '--impl', 'reference', '--scale', '8', '--frames', '3', '--steps', '1',
            '--warmup', '1']
import bench
bench.main()
maps = open('/proc/self/maps').read()
print('MAPS', 'libav1b.so' in maps, 'libav1synth.so' in maps, 'libav1ref.so' in maps)
'''


def test_reference_arm_maps_only_the_oracle(oracle):
    r = subprocess.run([sys.executable, '-c', PROBE], capture_output=True, text=True, cwd=ROOT,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line['impl'] == 'reference' and line['value'] > 0
    assert line['config']['gop'] == '1 key + 2 inter' and line['config']['frames_per_step'] == 3
    assert line['cpu_baseline']['kind'] == 'reference'
    assert line['e2e']['h2d_bytes_per_step'] == 0
    assert lines[1] == 'MAPS False False True'


def test_both_arms_name_the_same_config():
    sys.path.insert(0, ROOT)
    import bench
    a = bench.config_dict(3840, 2160, 2880, 30, 1)
    assert a['gop'] == '1 key + 29 inter' and a['seed'] == bench.SEED
    assert 'film grain' in a['workload']
