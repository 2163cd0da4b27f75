"""The served form (av1b_server_*): streams admitted by the device memory
they need, frame requests planned as they arrive and run in continuously
batched steps. Each stream's frames must come out the same as when the
stream is decoded alone (through the single-stream path, which the parity
tests pin to the oracle), whatever else is in the mix and whenever its
requests arrive."""
import ctypes
import random
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def spec(av1b):
    A = av1b
    return [
        # (width, height, coded_width, bit_depth, sb, tools, key_interval, max_refs)
        (160, 96, 0, 8, 64, A.TOOLS_ALL, 30, 2),
        (240, 136, 0, 10, 64, A.TOOLS_ALL, 30, 3),
        (480, 270, 360, 10, 128, A.TOOLS_ALL, 30, 3),
        (192, 128, 0, 12, 64, A.TOOLS_ALL, 3, 3),
        (150, 90, 0, 8, 64, A.TOOLS_ALL | A.TOOL_INTERINTRA | A.TOOL_INTRABC, 30, 3),
    ]


FRAMES = 6


def blobs_of(av1b, i, prm):
    return [av1b.synth_frame_ex(*prm[:6], 700 + i, k, prm[6], max_refs=prm[7]) for k in range(FRAMES)]


def pitch_of(w):
    return (w + 63) & ~63


@pytest.fixture(scope='module')
def solo(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    import refdec
    out = []
    for i, prm in enumerate(spec(av1b)):
        dec = av1b.Decoder(0)
        st = refdec.Stream(dec, max_refs=prm[7])
        nv = []
        for k, b in enumerate(blobs_of(av1b, i, prm)):
            slot, _ = st.decode(k, b, read_back=False)
            nv.append(dec.to_nv12(slot, pitch_of(prm[0]), prm[0], prm[1]))
        dec.close()
        out.append(nv)
    return out


def d2h(ptr, n):
    rt = ctypes.CDLL('libcudart.so')
    a = np.empty(n, dtype=np.uint8)
    assert rt.cudaMemcpy(ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(ptr), ctypes.c_size_t(n), 2) == 0
    return a


def test_served_frames_match_solo(av1b, solo):
    """Requests of all streams arrive interleaved in a random order (each
    stream's in its own order) with random gaps; every result's NV12 equals
    the stream's solo decode, and its timing fields are consistent."""
    sp = spec(av1b)
    srv = av1b.Server(0, max_inflight=2, planner_threads=4)
    ids = []
    for prm in sp:
        sid, hbm = srv.open(prm[0], prm[1], prm[3], coded_width=prm[2], max_refs=prm[7],
                            nv12_pitch=pitch_of(prm[0]))
        assert hbm > 0
        ids.append(sid)
    blobs = [blobs_of(av1b, i, prm) for i, prm in enumerate(sp)]
    order = [i for i in range(len(sp)) for _ in range(FRAMES)]
    random.Random(3).shuffle(order)
    nxt = [0] * len(sp)
    got = {}
    rng = random.Random(5)
    for i in order:
        k = nxt[i]
        nxt[i] += 1
        srv.submit(ids[i], blobs[i][k], tag=1000 * i + k)
        time.sleep(rng.random() * 0.002)
        for r in srv.poll():
            got[(r.stream_id, r.frame_index)] = (r.status, d2h(r.nv12_device, r.nv12_bytes), r)
    srv.drain(60000)
    for r in srv.poll(1024):
        got[(r.stream_id, r.frame_index)] = (r.status, d2h(r.nv12_device, r.nv12_bytes), r)
    assert len(got) == len(sp) * FRAMES
    multi = 0
    for i, sid in enumerate(ids):
        for k in range(FRAMES):
            status, nv, r = got[(sid, k)]
            assert status == 0, (i, k, status)
            assert r.tag == 1000 * i + k
            assert r.done_ms >= r.arrival_ms and r.latency_ms > 0
            assert np.array_equal(nv, solo[i][k]), 'stream %d frame %d' % (i, k)
            multi += r.batch_size > 1
    assert multi > 0   # some frames ran together with other streams' frames
    st = srv.stats()
    assert st.completed == st.submitted == len(sp) * FRAMES
    srv.close()


def test_admission_is_gated_by_hbm(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    one = av1b.lib().av1b_stream_hbm_estimate(1920, 1080, 0, 10, 1, 1, 4, 8)
    assert one > 0
    srv = av1b.Server(0, hbm_budget=int(one * 2.5) + 8 * 3110400)
    a, _ = srv.open(1920, 1080, 10, max_refs=3, nv12_pitch=1920)
    b, _ = srv.open(1920, 1080, 10, max_refs=3, nv12_pitch=1920)
    with pytest.raises(av1b.Av1bError) as e:
        srv.open(1920, 1080, 10, max_refs=3, nv12_pitch=1920)
    assert e.value.code == -3
    srv.close_stream(a)
    c, _ = srv.open(1920, 1080, 10, max_refs=3, nv12_pitch=1920)   # admitted once room is back
    assert srv.stats().streams == 2
    srv.close()


def test_a_bad_request_fails_alone(av1b, solo):
    """A frame whose reference lies before its stream's first frame fails at
    planning with a syntax error; the other streams' frames are unaffected."""
    sp = spec(av1b)[:2]
    srv = av1b.Server(0)
    ids = [srv.open(p[0], p[1], p[3], coded_width=p[2], max_refs=p[7], nv12_pitch=pitch_of(p[0]))[0]
           for p in sp]
    good = blobs_of(av1b, 0, sp[0])
    bad = blobs_of(av1b, 1, sp[1])[1]    # an inter frame submitted as the stream's first
    srv.submit(ids[1], bad)
    for k in range(3):
        srv.submit(ids[0], good[k])
    srv.drain(60000)
    res = {(r.stream_id, r.frame_index): r for r in srv.poll(64)}
    assert res[(ids[1], 0)].status == -4
    for k in range(3):
        r = res[(ids[0], k)]
        assert r.status == 0
        assert np.array_equal(d2h(r.nv12_device, r.nv12_bytes), solo[0][k])
    srv.close()
