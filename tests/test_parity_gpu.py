"""GPU parity: the CUDA path against the oracle (the reference's own CPU
backend) on the same seeded FrameSyntax, sample for sample, and against the
committed golden hashes. Every comparison is exact: the path is integer."""
import numpy as np
import pytest

import golden_util

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def dec(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    d = av1b.Decoder(0)
    yield d
    d.close()


def first_mismatch(a, b):
    d = np.argwhere(a != b)
    if not len(d):
        return None
    y, x = d[0]
    return 'n=%d first (y=%d, x=%d) gpu=%d oracle=%d' % (len(d), y, x, a[y, x], b[y, x])


def run_pair(av1b, refdec, dec, params, n, seed=4242, check_outputs=True):
    """Decodes n frames of a generated stream with both decoders and compares
    the planes of every frame; the NV12 and RGB packs of the newest and an
    older slot at the end."""
    ref = refdec.RefDecoder()
    sg, sr = refdec.Stream(dec), refdec.Stream(ref)
    w, h = params[0], params[1]
    for k in range(n):
        b = av1b.synth_frame_ex(*params[:6], seed, k, params[6])
        _, pg = sg.decode(k, b)
        _, pr = sr.decode(k, b)
        for p in range(3):
            mm = first_mismatch(pg[p], pr[p])
            assert mm is None, 'frame %d plane %d: %s' % (k, p, mm)
    if check_outputs:
        pitch = (w + 63) & ~63
        for k in (n - 1, max(0, n - 2)):
            a = dec.to_nv12(sg.slots[k], pitch, w, h)
            b = ref.to_nv12(sr.slots[k], pitch, w, h)
            assert np.array_equal(a, b), 'NV12 of frame %d' % k
        a = dec.to_rgb(sg.slots[n - 1], 1, 0, w, h)
        b = ref.to_rgb(sr.slots[n - 1], 1, 0, w, h)
        assert np.array_equal(a, b), 'RGB'
    for s in list(sg.slots.values()):
        dec.release_reference(s)


def stage_cases(av1b):
    A = av1b
    nodb = A.TOOL_NO_DEBLOCK | A.TOOL_NO_CDEF
    intra = A.TOOL_TX64 | A.TOOL_ALLTYPES | A.TOOL_CFL | A.TOOL_PALETTE | A.TOOL_FILTER_INTRA | \
        A.TOOL_EDGE_VARIANTS
    inter = A.TOOL_TX64 | A.TOOL_ALLTYPES | A.TOOL_COMPOUND | A.TOOL_MASKS | A.TOOL_OBMC | A.TOOL_WARP
    return {
        'intra_itx_8bit': ((160, 96, 0, 8, 64, nodb, 0), 1),
        'inter_8bit': ((160, 96, 0, 8, 64, nodb, 0), 3),
        'deblock_8bit': ((160, 96, 0, 8, 64, A.TOOL_NO_CDEF, 0), 3),
        'config1_small': ((160, 96, 0, 8, 64, 0, 0), 4),
        'odd_size': ((150, 90, 0, 8, 64, 0, 0), 3),
        'intra_tools_10bit': ((240, 136, 0, 10, 64, intra | nodb, 30), 1),
        'inter_tools_10bit': ((240, 136, 0, 10, 64, inter | nodb, 30), 4),
        'all_no_lr_grain': ((240, 136, 0, 10, 64, A.TOOLS_ALL & ~(A.TOOL_LR | A.TOOL_GRAIN), 30), 4),
        'loop_restoration': ((240, 136, 0, 10, 64, A.TOOLS_ALL & ~A.TOOL_GRAIN, 30), 3),
        'film_grain': ((240, 136, 0, 10, 64, A.TOOLS_ALL, 30), 3),
        'superres_128sb': ((480, 270, 360, 10, 128, A.TOOLS_ALL, 30), 3),
        'odd_superres_grain': ((150, 90, 112, 10, 64, A.TOOLS_ALL, 30), 2),
        'interintra_intrabc_residual': ((240, 136, 0, 10, 64, A.TOOLS_ALL | A.TOOL_INTERINTRA |
                                         A.TOOL_INTRABC | A.TOOL_RESIDUAL, 30), 4),
        'lossless': ((160, 96, 0, 8, 64, A.TOOL_LOSSLESS, 0), 2),
        'bitdepth_12': ((192, 128, 0, 12, 64, A.TOOLS_ALL, 30), 2),
        'tiny_16x16': ((16, 16, 0, 8, 64, A.TOOLS_ALL, 30), 3),
        'key_interval_2': ((128, 72, 0, 10, 64, A.TOOLS_ALL, 2), 5),
    }


CASES = ['intra_itx_8bit', 'inter_8bit', 'deblock_8bit', 'config1_small', 'odd_size',
         'intra_tools_10bit', 'inter_tools_10bit', 'all_no_lr_grain', 'loop_restoration',
         'film_grain', 'superres_128sb', 'odd_superres_grain', 'interintra_intrabc_residual', 'lossless', 'bitdepth_12',
         'tiny_16x16', 'key_interval_2']


@pytest.mark.parametrize('name', CASES)
def test_stage_parity(av1b, oracle, dec, name):
    params, n = stage_cases(av1b)[name]
    run_pair(av1b, oracle, dec, params, n)


@pytest.mark.parametrize('config,scale,frames', [(1, 2, 3), (2, 2, 3), (3, 4, 3)])
def test_config_parity_reduced(av1b, oracle, dec, config, scale, frames):
    """The three workloads at a reduced size, through av1b_synth_frame."""
    ref = oracle.RefDecoder()
    sg, sr = oracle.Stream(dec), oracle.Stream(ref)
    for k in range(frames):
        b = av1b.synth_frame(config, scale, 99, k)
        _, pg = sg.decode(k, b)
        _, pr = sr.decode(k, b)
        for p in range(3):
            assert first_mismatch(pg[p], pr[p]) is None, (k, p)
    for s in list(sg.slots.values()):
        dec.release_reference(s)


def test_masks_predicted_or_shared(av1b, oracle):
    """Chroma blocks of difference-weighted compounds: reading the luma
    block's mask (the default) and predicting the luma they cover in the full
    kernel (sharing off) both match the oracle."""
    params, n = stage_cases(av1b)['inter_tools_10bit']
    for share in (False, True):
        d = av1b.Decoder(0)
        d.set_shared_masks(share)
        run_pair(av1b, oracle, d, params, n, seed=77, check_outputs=False)
        d.close()


def test_golden_hashes(av1b, dec):
    """Against the committed fixtures: works without the oracle build."""
    for case in golden_util.load():
        got = golden_util.run_case(dec, case, av1b)
        assert got == case['frames'], case['name']
        dec.reset()


def test_full_size_4k_superres_parity(av1b, oracle, dec):
    """Config 3 at its full size (coded 2880x2160 -> 3840x2160, 10-bit), the key
    frame and two inter frames, against the oracle."""
    ref = oracle.RefDecoder()
    sg, sr = oracle.Stream(dec), oracle.Stream(ref)
    for k in range(3):
        b = av1b.synth_frame(3, 1, 5, k)
        _, pg = sg.decode(k, b)
        _, pr = sr.decode(k, b)
        for p in range(3):
            assert first_mismatch(pg[p], pr[p]) is None, (k, p)
    a = dec.to_nv12(sg.slots[2], 4096, 3840, 2160)
    b = ref.to_nv12(sr.slots[2], 4096, 3840, 2160)
    assert np.array_equal(a, b)
    for s in list(sg.slots.values()):
        dec.release_reference(s)


def test_planned_decode_matches_direct(av1b, dec):
    """plan_frame + decode_reference_planned gives the direct decode's pixels,
    also when the frames are queued without waiting."""
    blobs = [av1b.synth_frame(2, 8, 31, k) for k in range(4)]
    w, _, h, _, sx, sy = blobs[0].header
    shapes = av1b.plane_shapes(w, h, sx, sy)
    import refdec
    direct = refdec.Stream(dec)
    want = [direct.decode(k, b)[1] for k, b in enumerate(blobs)]
    for s in list(direct.slots.values()):
        dec.release_reference(s)
    ring = [dec.reserve_reference() for _ in range(4)]
    plans = []
    for k, b in enumerate(blobs):
        d = b.get_refs()
        b.set_refs([ring[(k - x) % 4] for x in d])
        plans.append(dec.plan(b))
        b.set_refs(d)
    got = []
    for k, pl in enumerate(plans):
        planes = [np.empty(s, dtype=np.uint16) for s in shapes]
        dec.decode_planned(pl, slot=ring[k % 4], keep=True, wait=False, planes=planes)
        got.append(planes)
    dec.sync()
    for k in range(4):
        for p in range(3):
            assert np.array_equal(got[k][p], want[k][p]), (k, p)
    for pl in plans:
        dec.free_plan(pl)
    for s in ring:
        dec.release_reference(s)


def test_planning_on_other_threads(av1b, dec):
    """Two planner threads plan frames k + 1 .. k + 3 (validation, records,
    uploads) while frame k decodes and packs NV12 on the calling thread - the
    pipelined use of plan_frame / decode_reference_planned, with two planners
    of the decoder busy at once - and every frame's NV12 equals the one-call
    decode's. Plans are recycled through the decoder's pool."""
    from concurrent.futures import ThreadPoolExecutor
    blobs = [av1b.synth_frame(2, 4, 77, k) for k in range(10)]
    w, _, h, _, sx, sy = blobs[0].header
    pitch = (w + 63) // 64 * 64
    import refdec
    direct = refdec.Stream(dec)
    want = []
    for k, b in enumerate(blobs):
        slot, _ = direct.decode(k, b, read_back=False)
        want.append(dec.to_nv12(slot, pitch, w, h))
    for s in list(direct.slots.values()):
        dec.release_reference(s)
    ring = [dec.reserve_reference() for _ in range(4)]

    def plan(k):
        b = blobs[k]
        d = b.get_refs()
        b.set_refs([ring[(k - x) % 4] for x in d])
        try:
            return dec.plan(b)
        finally:
            b.set_refs(d)

    ahead = 3
    with ThreadPoolExecutor(max_workers=2) as ex:
        futs = {k: ex.submit(plan, k) for k in range(ahead)}
        for k in range(len(blobs)):
            pl = futs.pop(k).result(timeout=120)
            if k + ahead < len(blobs):
                futs[k + ahead] = ex.submit(plan, k + ahead)
            dec.decode_planned(pl, slot=ring[k % 4], keep=True, wait=False)
            got = dec.to_nv12(ring[k % 4], pitch, w, h)
            dec.free_plan(pl)
            assert np.array_equal(got, want[k]), k
        dec.sync()
    for s in ring:
        dec.release_reference(s)


def test_decode_drop_and_slot_semantics(av1b, oracle, dec):
    """decode (keep = False) holds no slot; to_nv12 of an older slot packs its
    stored picture (before film grain), of the newest the output picture."""
    b0 = av1b.synth_frame(2, 8, 8, 0)
    b1 = av1b.synth_frame(2, 8, 8, 1)
    w, _, h, _, _, _ = b0.header
    ref = oracle.RefDecoder()
    s0g, _ = dec.decode(b0)
    s0r, _ = ref.decode(b0)
    b1.set_refs([s0g])
    dec.decode(b1, keep=False)
    b1.set_refs([s0r])
    ref.decode(b1, keep=False)
    pitch = (w + 63) & ~63
    assert np.array_equal(dec.to_nv12(s0g, pitch, w, h), ref.to_nv12(s0r, pitch, w, h))
    assert np.array_equal(dec.to_nv12(-1, pitch, w, h), ref.to_nv12(-1, pitch, w, h))
    dec.release_reference(s0g)


def test_errors_are_reported_not_faulted(av1b, dec):
    b = av1b.synth_frame(1, 8, 3, 1)
    b.set_refs([31])  # a slot that holds nothing
    with pytest.raises(av1b.Av1bError) as e:
        dec.decode(b)
    assert e.value.code == -4
    with pytest.raises(av1b.Av1bError):
        dec.to_nv12(0, 63, 160, 90)
    # the decoder is still usable
    slot, planes = dec.decode(av1b.synth_frame(1, 8, 3, 0))
    assert slot >= 0 and planes[0].shape == (90, 160)
    dec.release_reference(slot)


def test_invalid_records_name_the_first_one(av1b, oracle, dec):
    """Deblocking edges and CDEF blocks are validated on the device; an invalid
    one fails the frame with the message of the first invalid record in the
    frame's validation order (edges, then CDEF blocks, then restoration and
    film grain), and the decoder stays usable."""
    b = av1b.synth_frame(2, 8, 3, 0)

    def error_of(blob):
        with pytest.raises(av1b.Av1bError) as e:
            dec.decode(blob)
        assert e.value.code == -4
        return str(e.value)

    last = oracle.blob_counts(b)['deblock'] - 1
    assert 'deblock level out of range' in error_of(oracle.corrupt(b, oracle.CORRUPT_EDGE_LEVEL, last))
    assert 'outside the picture' in error_of(oracle.corrupt(b, oracle.CORRUPT_EDGE_OUTSIDE, 0))
    assert 'CDEF parameters' in error_of(oracle.corrupt(b, oracle.CORRUPT_CDEF_DIR, 5))
    both = oracle.corrupt(oracle.corrupt(b, oracle.CORRUPT_CDEF_DIR, 0), oracle.CORRUPT_EDGE_LEVEL, last)
    assert 'deblock level' in error_of(both)
    lr_and_cdef = oracle.corrupt(oracle.corrupt(b, oracle.CORRUPT_LR_UNIT), oracle.CORRUPT_CDEF_DIR, 7)
    assert 'CDEF parameters' in error_of(lr_and_cdef)
    assert 'restoration unit size' in error_of(oracle.corrupt(b, oracle.CORRUPT_LR_UNIT))
    assert 'film grain' in error_of(oracle.corrupt(b, oracle.CORRUPT_GRAIN))
    slot, planes = dec.decode(b)
    ref_slot, ref_planes = oracle.RefDecoder().decode(b)
    for p in range(3):
        assert np.array_equal(planes[p], ref_planes[p])
    dec.release_reference(slot)


def test_unit_trace_is_consistent(av1b, oracle, dec):
    """The opt-in phase B trace: every dependency-scheduled block of a key
    frame has a record, claimed <= ready <= published, and the dependency it
    names as published last was published before it became ready. Tracing
    changes no sample."""
    b = av1b.synth_frame(2, 4, 11, 0)
    slot0, plain = dec.decode(b)
    dec.release_reference(slot0)
    dec.set_unit_trace(True)
    try:
        slot, traced = dec.decode(b)
        tr = dec.unit_trace().astype(np.int64)
    finally:
        dec.set_unit_trace(False)
    dec.release_reference(slot)
    for p in range(3):
        assert np.array_equal(plain[p], traced[p])
    assert tr.shape == (oracle.blob_counts(b)['blocks'], 4)
    live = np.nonzero(tr[:, 2])[0]
    assert len(live) > 100          # a key frame: every block is in phase B
    assert np.all(tr[live, 0] <= tr[live, 1]) and np.all(tr[live, 1] <= tr[live, 2])
    who = tr[live, 3]
    named = who >= 0
    named &= who < len(tr)
    deps = who[named]
    assert np.all(tr[deps, 2] > 0)
    assert np.all(tr[deps, 2] <= tr[live[named], 1])


def test_bounded_wait_gives_up(dec):
    """A device wait on a flag nothing sets returns an error status after its
    limit instead of hanging (no fault, no trap)."""
    status, ms = dec.selftest_wait(2_000_000)  # 2 ms
    assert status == 1
    assert 1.0 < ms < 1000.0


def test_measured_peaks(av1b):
    """The roofs the stage report divides by: the integer-ALU peak and the
    floor of a dependency step (one flag handed between two SMs)."""
    assert av1b.int_peak(0, 0) > 1e12
    ns = av1b.handoff_peak(0)
    assert 50.0 < ns < 20000.0


def test_hbm_budget_is_enforced(av1b):
    d = av1b.Decoder(0, hbm_budget=1 << 20)
    with pytest.raises(av1b.Av1bError) as e:
        d.decode(av1b.synth_frame(1, 8, 1, 0))
    assert e.value.code == -3
    d.close()


def test_nv12_split_pack(av1b, oracle, dec):
    """nv12_pack_begin / wait / release (the reference's split pack,
    av1gpu.hpp:748-772): a pack begun right after a frame carries that frame's
    picture after film grain even when the next frame is decoded before the
    wait; a pack of an older slot carries its stored picture; several packs
    are outstanding at once; a view of the page-locked bytes and a copy agree."""
    w, h = 240, 136
    params = (w, h, 0, 10, 64, av1b.TOOLS_ALL, 30)
    ref = oracle.RefDecoder()
    sg, sr = oracle.Stream(dec), oracle.Stream(ref)
    pitch = 256
    pending = []
    for k in range(5):
        b = av1b.synth_frame_ex(*params[:6], 77, k, params[6])
        sg.decode(k, b, read_back=False)
        sr.decode(k, b, read_back=False)
        expect = ref.to_nv12(sr.slots[k], pitch, w, h)
        pending.append((dec.nv12_pack_begin(sg.slots[k], pitch), expect))
        if k >= 1:
            handle, want = pending.pop(0)
            got = dec.nv12_pack_wait(handle)
            assert np.array_equal(got, want), 'frame %d (packed before the next decode)' % (k - 1)
            copy = dec.nv12_pack_wait(handle, np.empty(want.size, dtype=np.uint8))
            assert np.array_equal(copy, want)
            dec.nv12_pack_release(handle)
    handle, want = pending.pop()
    assert np.array_equal(dec.nv12_pack_wait(handle), want)
    dec.nv12_pack_release(handle)
    older = [dec.nv12_pack_begin(sg.slots[k], pitch) for k in (3, 4)]
    for k, handle in zip((3, 4), older):
        assert np.array_equal(dec.nv12_pack_wait(handle), ref.to_nv12(sr.slots[k], pitch, w, h))
        dec.nv12_pack_release(handle)
    with pytest.raises(av1b.Av1bError):
        dec.nv12_pack_wait(older[0])
    for s in list(sg.slots.values()):
        dec.release_reference(s)


@pytest.mark.parametrize('name', [n for n, _ in golden_util.WORKLOADS])
def test_full_size_workload_hashes(av1b, dec, name):
    """The benchmark workloads at full size, every frame against the oracle's
    hashes (tests/golden/workloads.json): config 1 (1280x720 8-bit, 30
    frames), config 2 (1920x1080 10-bit, 60 frames, key frames at 0 and 30,
    three-slot compound) and the exact GOP bench.py times (config 3, its seed,
    30 frames)."""
    spec = dict(golden_util.WORKLOADS)[name]
    want = golden_util.load_workloads()[name]['frames']
    got = golden_util.run_workload(dec, spec, av1b)
    assert len(got) == len(want) == spec[2]
    for k, (g, w) in enumerate(zip(got, want)):
        assert g == w, '%s frame %d' % (name, k)


def test_deferred_grain_outputs(av1b, oracle, dec):
    """A planned decode that reads nothing back leaves the frame's film grain
    to its outputs: the NV12 pack applies it while packing, and the display
    picture is made when asked for (device planes, RGB); all equal the oracle."""
    import ctypes
    blobs = [av1b.synth_frame(2, 4, 61, k) for k in range(3)]
    w, _, h, _, sx, sy = blobs[0].header
    ref = oracle.RefDecoder()
    sr = oracle.Stream(ref)
    ring = [dec.reserve_reference() for _ in range(4)]
    rt = ctypes.CDLL('libcudart.so')
    pitch = (w + 63) & ~63
    for k, b in enumerate(blobs):
        d = b.get_refs()
        b.set_refs([ring[(k - x) % 4] for x in d])
        pl = dec.plan(b)
        b.set_refs(d)
        dec.decode_planned(pl, slot=ring[k], keep=True, wait=True)
        dec.free_plan(pl)
        # the oracle's frame k decoded now, so that it too is the frame decoded last
        rslot, rplanes = sr.decode(k, b)
        if k == 0:   # NV12 first: packed with the grain applied while packing
            assert np.array_equal(dec.to_nv12(ring[k], pitch, w, h), ref.to_nv12(rslot, pitch, w, h))
        if k == 1:   # planes first: the display picture is made on demand
            ptr = (ctypes.c_void_p * 3)()
            stride = (ctypes.c_int32 * 3)()
            assert av1b.lib().av1b_slot_planes_device(dec.h, ring[k], ptr, stride) == 0
            dec.sync()   # the display picture is made on the decoder's stream
            for p, (rows, cols) in enumerate(av1b.plane_shapes(w, h, sx, sy)):
                a = np.empty((rows, cols), dtype=np.uint16)
                assert rt.cudaMemcpy2D(ctypes.c_void_p(a.ctypes.data), ctypes.c_size_t(cols * 2),
                                       ctypes.c_void_p(ptr[p]), ctypes.c_size_t(stride[p] * 2),
                                       ctypes.c_size_t(cols * 2), ctypes.c_size_t(rows), 2) == 0
                assert np.array_equal(a, rplanes[p]), (k, p)
            assert np.array_equal(dec.to_nv12(ring[k], pitch, w, h), ref.to_nv12(rslot, pitch, w, h))
        if k == 2:   # RGB
            assert np.array_equal(dec.to_rgb(ring[k], 1, 0, w, h), ref.to_rgb(rslot, 1, 0, w, h))
    for s in ring:
        dec.release_reference(s)
