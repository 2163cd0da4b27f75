"""The planner's dependency schedule on the host (no GPU): tests/cpp/
plan_invariants.cu compiles the planner with plain host allocations and checks,
on seeded frames of five geometries, that every phase B block's dependencies
lie earlier in its own chain or in a chain claimed before it - the property
that lets the device's warps finish without a cooperative launch - and that
the records do not depend on the number of host threads, and that the
prediction tiles are grouped for the kernels that take them (the lean
kernel's unmasked and masked builds, the full kernel, the chroma tiles that
read a luma mask last) with every luma mask inside the frame's mask pool.
Builds with the chain admission check, or the tile grouping, broken in a copy
of the planner must fail the same checks."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, 'av1ongpu_b200', 'csrc')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')


def build_checker(tmp_path, src_dir=None, name='plan_invariants'):
    from av1ongpu_b200 import build as b
    b.build()
    objs = [os.path.join(b.OUT, f) for f in ('kernels.cu.o', 'plan_host.cpp.o', 'synth.cpp.o',
                                             'blob.cpp.o', 'api.cpp.o', 'noalloc.cu.o')]
    exe = str(tmp_path / name)
    inc = (['-I', src_dir] if src_dir else []) + ['-I', CSRC, '-I', os.path.join(ROOT, 'include')]
    cmd = [NVCC, '-gencode', 'arch=compute_100a,code=sm_100a', '-O2', '-std=c++17',
           '-diag-suppress', '68'] + inc + [os.path.join(ROOT, 'tests', 'cpp', 'plan_invariants.cu')] + \
        objs + ['-o', exe, '-lpthread']
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


@pytest.fixture(scope='module')
def have_nvcc():
    if not (os.path.exists(NVCC) or shutil.which('nvcc')):
        pytest.skip('nvcc not available')


def test_chains_only_wait_on_earlier_work(tmp_path, have_nvcc):
    exe = build_checker(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    assert r.stdout.strip().endswith('ok')
    assert 'FAIL' not in r.stdout


def test_checker_catches_an_unchecked_chain_admission(tmp_path, have_nvcc):
    src = open(os.path.join(CSRC, 'decoder.cu')).read()
    admission = 'ok &= hk[udeps[j]] <= hc;'
    assert src.count(admission) == 1
    bad = tmp_path / 'bad'
    bad.mkdir()
    (bad / 'decoder.cu').write_text(src.replace(admission, 'ok &= true;'))
    exe = build_checker(tmp_path, str(bad), 'plan_invariants_bad')
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert 'waits for' in r.stdout


def test_checker_catches_a_misgrouped_tile(tmp_path, have_nvcc):
    src = open(os.path.join(CSRC, 'decoder.cu')).read()
    grouping = '(r.mask_kind ? O->inter_tiles_mask : O->inter_tiles)'
    assert src.count(grouping) == 1
    bad = tmp_path / 'bad'
    bad.mkdir()
    (bad / 'decoder.cu').write_text(src.replace(grouping, 'O->inter_tiles'))
    exe = build_checker(tmp_path, str(bad), 'plan_invariants_badtiles')
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert 'in group 0, not 1' in r.stdout
