"""The batched form (av1b_batch_*): one frame of each of several independent
streams of different geometry, bit depth and tools decoded as one step of
persistent kernels. Every stream's output planes and NV12 pack must equal
its solo decode through the single-stream path - which the parity tests pin
to the oracle - sample for sample and byte for byte, whatever the launch
shape, with and without graph replay and with the film grain applied inside
the NV12 pack."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def streams_spec(av1b):
    A = av1b
    return [
        # (width, height, coded_width, bit_depth, sb, tools, key_interval)
        (160, 96, 0, 8, 64, 0, 0),
        (240, 136, 0, 10, 64, A.TOOLS_ALL, 30),
        (480, 270, 360, 10, 128, A.TOOLS_ALL, 30),          # superres + restoration + grain
        (150, 90, 0, 8, 64, A.TOOLS_ALL, 2),                 # odd size, a key frame every 2
        (192, 128, 0, 12, 64, A.TOOLS_ALL, 30),
        (240, 136, 0, 10, 64, A.TOOLS_ALL | A.TOOL_INTERINTRA | A.TOOL_INTRABC | A.TOOL_RESIDUAL, 30),
    ]


FRAMES = 4


class _Rt:
    def __init__(self):
        self.rt = ctypes.CDLL('libcudart.so')

    def d2h(self, dst, src, n):
        assert self.rt.cudaMemcpy(ctypes.c_void_p(dst), ctypes.c_void_p(src), ctypes.c_size_t(n), 2) == 0

    def d2h_2d(self, dst, dpitch, src, spitch, width, height):
        assert self.rt.cudaMemcpy2D(ctypes.c_void_p(dst), ctypes.c_size_t(dpitch), ctypes.c_void_p(src),
                                    ctypes.c_size_t(spitch), ctypes.c_size_t(width),
                                    ctypes.c_size_t(height), 2) == 0


def read_planes(av1b, rt, dec, slot, header):
    w, _, h, _, sx, sy = header
    ptr = (ctypes.c_void_p * 3)()
    stride = (ctypes.c_int32 * 3)()
    assert av1b.lib().av1b_slot_planes_device(dec.h, slot, ptr, stride) == 0
    dec.sync()   # a display picture left to the outputs is made on the decoder's stream
    out = []
    for p, (rows, cols) in enumerate(av1b.plane_shapes(w, h, sx, sy)):
        a = np.empty((rows, cols), dtype=np.uint16)
        rt.d2h_2d(a.ctypes.data, cols * 2, ptr[p], stride[p] * 2, cols * 2, rows)
        out.append(a)
    return out


@pytest.fixture(scope='module')
def solo(av1b):
    """Every stream decoded alone, frame by frame: planes and NV12."""
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    import refdec
    out = []
    for k_s, prm in enumerate(streams_spec(av1b)):
        dec = av1b.Decoder(0)
        st = refdec.Stream(dec)
        frames = []
        for k in range(FRAMES):
            b = av1b.synth_frame_ex(*prm[:6], 900 + k_s, k, prm[6])
            slot, planes = st.decode(k, b)
            pitch = (prm[0] + 63) & ~63
            frames.append((planes, dec.to_nv12(slot, pitch, prm[0], prm[1])))
        dec.close()
        out.append(frames)
    return out


def run_batched(av1b, solo, config=None, fuse=False, graph=True, share_masks=True):
    import torch
    rt = _Rt()
    spec = streams_spec(av1b)
    batch = av1b.Batch(0)
    c = batch.config()
    if config:
        for k, v in config.items():
            setattr(c, k, v)
    c.fuse_grain_nv12 = 1 if fuse else 0
    c.use_graph = 1 if graph else 0
    batch.set_config(c)
    decs = [av1b.Decoder(0) for _ in spec]
    for d in decs:
        d.set_shared_masks(share_masks)
    rings = [[d.reserve_reference() for _ in range(4)] for d in decs]
    nv_bufs = []
    for prm in spec:
        pitch = (prm[0] + 63) & ~63
        n = av1b.nv12_size(prm[0], prm[1], 1, 1, pitch)
        nv_bufs.append((torch.zeros(n, dtype=torch.uint8, device='cuda:0'), pitch, n))
    for k in range(FRAMES):
        plans = []
        blobs = []
        for i, prm in enumerate(spec):
            b = av1b.synth_frame_ex(*prm[:6], 900 + i, k, prm[6])
            d = b.get_refs()
            b.set_refs([rings[i][(k - x) % 4] for x in d])
            plans.append(decs[i].plan(b))
            b.set_refs(d)
            blobs.append(b)
        got = batch.decode(decs, plans, slots=[r[k % 4] for r in rings],
                           nv12=[(t.data_ptr(), p, n) for t, p, n in nv_bufs])
        assert got == [r[k % 4] for r in rings]
        batch.sync()
        for i, prm in enumerate(spec):
            want_planes, want_nv = solo[i][k]
            planes = read_planes(av1b, rt, decs[i], got[i], blobs[i].header)
            for p in range(3):
                assert np.array_equal(planes[p], want_planes[p]), \
                    'stream %d frame %d plane %d (fuse=%s graph=%s)' % (i, k, p, fuse, graph)
            t, pitch, n = nv_bufs[i]
            nv = t.cpu().numpy()
            assert np.array_equal(nv, want_nv), 'stream %d frame %d NV12' % (i, k)
            # the decoder's own output call after the step agrees
            assert np.array_equal(decs[i].to_nv12(got[i], pitch, prm[0], prm[1]), want_nv)
        for i, pl in enumerate(plans):
            decs[i].free_plan(pl)
    for d in decs:
        d.close()
    batch.close()


def test_batched_step_matches_solo(av1b, solo):
    run_batched(av1b, solo)


def test_batched_step_without_graph_and_with_grain_in_pack(av1b, solo):
    run_batched(av1b, solo, fuse=True, graph=False)
    run_batched(av1b, solo, fuse=True, graph=True)


def test_batched_step_with_chroma_masks_predicted(av1b, solo):
    """Chroma blocks of difference-weighted compounds predicting the luma they
    cover (the full kernel's stage) instead of reading their luma block's
    mask: the same frames as the solo decodes, which read the masks."""
    run_batched(av1b, solo, share_masks=False)


def test_batched_step_launch_shapes(av1b, solo):
    """The smallest launch (one CTA an SM everywhere) and large claims: the
    persistent kernels loop over many items per CTA and warp."""
    ones = (ctypes.c_int32 * 24)(*([1] * 24))
    run_batched(av1b, solo, config={'ctas_per_sm': ones, 'claim_chunk': 8})


def test_autotune_and_cache(av1b, tmp_path):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    spec = streams_spec(av1b)[:3]
    batch = av1b.Batch(0)
    decs = [av1b.Decoder(0) for _ in spec]
    rings = [[d.reserve_reference() for _ in range(2)] for d in decs]
    plans = []
    for i, prm in enumerate(spec):
        b0 = av1b.synth_frame_ex(*prm[:6], 5, 0, prm[6])
        s0, _ = decs[i].decode(b0)
        b1 = av1b.synth_frame_ex(*prm[:6], 5, 1, prm[6])
        b1.set_refs([s0 for _ in b1.get_refs()])
        plans.append(decs[i].plan(b1))
    cache = str(tmp_path / 'tune.txt')
    cfg, ms = batch.autotune(decs, plans, slots=[r[0] for r in rings], cache_path=cache, reps=1)
    assert ms > 0 and cfg['claim_chunk'] >= 1
    assert all(1 <= c <= 64 for c in cfg['ctas_per_sm'])
    text = open(cache).read()
    assert text.count('\n') == 1 and '\t' in text
    again = av1b.Batch(0)
    cfg2, ms2 = again.autotune(decs, plans, slots=[r[0] for r in rings], cache_path=cache, reps=1)
    assert ms2 == -1.0 and cfg2['ctas_per_sm'] == cfg['ctas_per_sm']
    for i, pl in enumerate(plans):
        decs[i].free_plan(pl)
    for d in decs:
        d.close()
    batch.close()
    again.close()


def test_batch_refuses_bad_steps(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    batch = av1b.Batch(0)
    d = av1b.Decoder(0)
    b = av1b.synth_frame(1, 8, 3, 0)
    pl = d.plan(b)
    with pytest.raises(av1b.Av1bError):
        batch.decode([d, d], [pl, pl])          # a decoder twice in one step
    with pytest.raises(av1b.Av1bError):
        batch.decode([d], [pl], nv12=[(1, 63, 10)])   # odd pitch
    d.free_plan(pl)
    d.close()
    batch.close()
