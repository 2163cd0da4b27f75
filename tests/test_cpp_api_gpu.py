"""The C++ drop-in API (include/av1gpu/av1gpu.hpp) used by a compiled client,
against the oracle on the same frames."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_client(tmp_path):
    exe = str(tmp_path / 'api_client')
    cmd = ['/usr/bin/g++', '-std=c++17', '-O1', os.path.join(ROOT, 'tests', 'cpp', 'api_client.cpp'),
           '-I', os.path.join(ROOT, 'include'), '-I', os.path.join(ROOT, 'av1ongpu_b200', 'csrc'),
           '-L', os.path.join(ROOT, 'av1ongpu_b200'), '-lav1b', '-lav1synth',
           '-Wl,-rpath,' + os.path.join(ROOT, 'av1ongpu_b200'), '-o', exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_cpp_client_matches_oracle(av1b, oracle, tmp_path):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    exe = build_client(tmp_path)
    params = (240, 136, 0, 10, 64, av1b.TOOLS_ALL)
    frames = 5
    out = str(tmp_path / 'out.bin')
    r = subprocess.run([exe, out] + [str(v) for v in params] + ['77', str(frames)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    data = open(out, 'rb').read()
    ref = oracle.RefDecoder()
    st = oracle.Stream(ref)
    w, h = params[0], params[1]
    pitch = (w + 63) & ~63
    pos = 0
    for k in range(frames):
        b = av1b.synth_frame_ex(*params, 77, k, 30)
        slot, planes = st.decode(k, b)
        for p in planes:
            n = p.size * 2
            got = np.frombuffer(data[pos:pos + n], dtype=np.uint16).reshape(p.shape)
            pos += n
            assert np.array_equal(got, p), 'frame %d' % k
        nv = ref.to_nv12(slot, pitch, w, h)
        got = np.frombuffer(data[pos:pos + nv.size], dtype=np.uint8)
        pos += nv.size
        assert np.array_equal(got, nv), 'nv12 frame %d' % k
    assert pos == len(data)
