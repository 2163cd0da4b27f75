"""CPU tests: the C ABI library, the syntax format, the workload generator and
the oracle (which is pinned here against the reference's own tests)."""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header='av1b.h', macro='AV1B_API', prefix='av1b_'):
    text = open(os.path.join(ROOT, 'include', header)).read()
    return sorted(set(re.findall(r'%s\s+[\w\s\*]*?\b(%s\w+)\s*\(' % (macro, prefix), text)))


def test_library_exports_every_declared_symbol(av1b):
    lib = av1b.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n


def test_generator_library_exports_every_declared_symbol(av1b):
    lib = av1b.synth_lib()
    names = declared_symbols('av1b_synth.h', 'AV1S_API', 'av1s_')
    assert len(names) == 4
    for n in names:
        assert hasattr(lib, n), n
    # the generator is host code apart from the decoder: it links no CUDA
    deps = subprocess.run(['ldd', av1b.SYNTH_LIB_PATH], capture_output=True, text=True).stdout
    assert 'cuda' not in deps and 'av1b' not in deps


def test_python_binds_every_exported_entry(av1b):
    assert set(av1b.exported_symbols()) <= set(declared_symbols())
    assert set(av1b.synth_exported_symbols()) == set(
        declared_symbols('av1b_synth.h', 'AV1S_API', 'av1s_'))


def test_synth_is_deterministic(av1b):
    a = av1b.synth_frame(2, 8, 123, 3).to_bytes()
    b = av1b.synth_frame(2, 8, 123, 3).to_bytes()
    c = av1b.synth_frame(2, 8, 124, 3).to_bytes()
    assert a == b
    assert a != c


def test_blob_view_and_refs(av1b):
    b = av1b.synth_frame(1, 8, 7, 2)
    w, cw, h, bd, sx, sy = b.header
    assert (w, h, bd, sx, sy) == (160, 90, 8, 1, 1)
    assert b.get_refs() == [1]
    b.set_refs([5])
    assert b.get_refs() == [5]
    # the library reads the list the Python header code wrote, and the reverse
    buf = (ctypes.c_int32 * 8)()
    assert av1b.lib().av1b_blob_get_refs(b.ptr, b.size, buf, 8) == 1 and buf[0] == 5
    assert av1b.lib().av1b_blob_set_refs(b.ptr, b.size, (ctypes.c_int32 * 2)(3, 9), 2) == 0
    assert b.get_refs() == [3, 9]
    b.set_refs([5])
    view = ctypes.create_string_buffer(4096)
    assert av1b.lib().av1b_syntax_view(b.ptr, b.size, view) == 0
    # a truncated buffer is refused
    assert av1b.lib().av1b_syntax_view(b.ptr, 40, view) != 0
    # the copy survives a round trip through bytes
    c = av1b.Blob.from_bytes(b.to_bytes())
    assert c.header == b.header and c.get_refs() == [5]


@pytest.mark.parametrize('config,scale', [(1, 1), (2, 1), (3, 4)])
def test_workload_shapes(av1b, config, scale):
    b = av1b.synth_frame(config, scale, 1, 0)
    w, cw, h, bd, sx, sy = b.header
    want = {1: (1280, 0, 720, 8), 2: (1920, 0, 1080, 10), 3: (960, 720, 540, 10)}[config]
    assert (w, cw, h, bd) == want


def test_nv12_size_rules(av1b):
    # nv12_buffer_size (factory.cpp:236-244): 4:2:0 only, even pitch >= chroma row
    assert av1b.nv12_size(64, 48, 1, 1, 64) == 64 * 72
    assert av1b.nv12_size(63, 47, 1, 1, 64) == 64 * (47 + 24)
    assert av1b.nv12_size(64, 48, 1, 1, 63) == 0
    assert av1b.nv12_size(64, 48, 1, 1, 62) == 0
    assert av1b.nv12_size(64, 48, 0, 0, 64) == 0


def test_decoder_refuses_without_device(av1b):
    if av1b.cuda_available():
        pytest.skip('a CUDA device is visible')
    with pytest.raises(av1b.Av1bError) as e:
        av1b.Decoder(0)
    assert e.value.code == -7


def test_oracle_reference_unit_tests(oracle):
    """The reference's own test_kernels / test_pipeline, built from its sources
    against the oracle's objects (oracle/Makefile `tests`)."""
    for name, checks in (('test_kernels', 2353), ('test_pipeline', 72)):
        exe = os.path.join(ROOT, 'oracle', '_ref', name)
        if not os.path.exists(exe):
            pytest.skip('%s not built (make -C oracle tests)' % name)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-2000:]
        m = re.search(r'%s: (\d+) checks, (\d+) failure' % name, r.stdout)
        assert m and int(m.group(1)) >= checks and int(m.group(2)) == 0


def test_oracle_matches_golden(oracle, av1b):
    """The oracle reproduces the committed golden hashes (tests/golden)."""
    import golden_util
    cases = golden_util.load()
    for case in cases[:4]:
        got = golden_util.run_case(oracle.RefDecoder(), case, av1b)
        assert got == case['frames'], case['name']


def test_batch_config_lists_every_stage(av1b):
    """The launch shape's dictionary view has one entry per stage of the
    batched step, the stages the header counts."""
    import re
    header = open(os.path.join(ROOT, 'include', 'av1b.h')).read()
    n = int(re.search(r'stages in launch order, (\d+) of them', header).group(1))
    assert len(av1b.Batch.STAGES) == n
    assert len(av1b.BatchConfig().as_dict()['ctas_per_sm']) == n
