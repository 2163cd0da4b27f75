"""The CUDA path on real streams: every frame of the reference's 24 bit-exact
test streams (intra and inter, 8/10/12 bit, 4:2:0/4:2:2/4:4:4, palette, intra
block copy, local warp and OBMC, inter-intra and wedges, segmentation,
superres, film grain, loop restoration, lossless, odd sizes, multi-tile),
replayed from the fixtures oracle/stream_dump made with the reference's own
front end, must hash to the dav1d frame hashes the reference's stream tests
check (CMakeLists.txt:272-350 of the reference). On a mismatch the oracle
replays the same stream and the message names the first differing sample."""
import numpy as np
import pytest

import stream_replay as sr

pytestmark = pytest.mark.gpu

NAMES = sr.fixture_names()


@pytest.fixture(scope='module')
def dec(av1b):
    if not av1b.cuda_available():
        pytest.skip('no CUDA device')
    d = av1b.Decoder(0)
    yield d
    d.close()


def first_difference(fx, dec, oracle):
    _, mine = sr.replay(fx, dec, keep_pictures=True)
    _, ref = sr.replay(fx, oracle.RefDecoder(), keep_pictures=True)
    for k, (a, b) in enumerate(zip(mine, ref)):
        for p in range(3):
            d = np.argwhere(a[p] != b[p])
            if len(d):
                y, x = d[0]
                return 'decode %d plane %d: %d samples differ, first (y=%d, x=%d) gpu=%d oracle=%d' % (
                    k, p, len(d), y, x, a[p][y, x], b[p][y, x])
    return 'the pictures agree with the oracle; the hash lists differ'


@pytest.mark.parametrize('name', NAMES or ['none'])
def test_stream_matches_recorded_hashes(av1b, dec, oracle, name):
    if not NAMES:
        pytest.skip('no stream fixtures (make -C oracle streams)')
    fx = sr.Fixture(name)
    got, _ = sr.replay(fx, dec)
    assert len(got) == len(fx.hashes), '%s: %d shown frames, %d hashes' % (
        name, len(got), len(fx.hashes))
    if got != fx.hashes:
        bad = [i for i, (a, b) in enumerate(zip(got, fx.hashes)) if a != b]
        pytest.fail('%s: shown frames %s differ; %s' % (name, bad[:8],
                                                       first_difference(fx, dec, oracle)))


@pytest.mark.parametrize('name', sr.fixture_names(levels=True) or ['none'])
def test_stream_from_levels_matches_recorded_hashes(av1b, dec, oracle, name):
    """The same streams as the reference pipeline hands a device dequantiser:
    coded levels, per-transform steps and QM offsets, no coefficient pool. The
    rasters are built on the device (k_dequant) and must give the same frames."""
    if not sr.fixture_names(levels=True):
        pytest.skip('no stream fixtures (make -C oracle streams)')
    fx = sr.Fixture(name, levels=True)
    got, _ = sr.replay(fx, dec)
    assert len(got) == len(fx.hashes)
    if got != fx.hashes:
        bad = [i for i, (a, b) in enumerate(zip(got, fx.hashes)) if a != b]
        pytest.fail('%s (levels): shown frames %s differ; %s' % (
            name, bad[:8], first_difference(sr.Fixture(name), dec, oracle)))


@pytest.mark.parametrize('name', ['lr_10bit', 'aom_444_10bit_320x240', 'lw_t2', 'tiles_grid'])
def test_quantiser_matrices_on_device(av1b, dec, oracle, name):
    """No test stream codes quantiser matrices, so they are planted: every
    coded transform of a levels stream gets a seeded matrix out of a seeded
    pool. The CUDA path dequantises the levels on the device; the oracle
    decodes the same frames expanded by the reference front end's own host
    dequantiser. Every picture must agree."""
    if name not in sr.fixture_names(levels=True):
        pytest.skip('no stream fixtures (make -C oracle streams)')
    fx = sr.Fixture(name, levels=True)
    pairs = {}

    def pair(k, payload):
        if k not in pairs:
            pairs[k] = oracle.dequant_pair(payload, 1000 + k)
        return pairs[k]

    _, mine = sr.replay(fx, dec, keep_pictures=True, rewrite=lambda k, p: pair(k, p)[0])
    _, ref = sr.replay(fx, oracle.RefDecoder(), keep_pictures=True,
                       rewrite=lambda k, p: pair(k, p)[1])
    assert len(mine) == len(ref)
    for k, (a, b) in enumerate(zip(mine, ref)):
        for p in range(3):
            d = np.argwhere(a[p] != b[p])
            assert not len(d), '%s decode %d plane %d: %d samples differ, first %s' % (
                name, k, p, len(d), tuple(d[0]))


STAGES = {
    'reconstruction': 15,      # prediction and residual only
    'deblock': 14,             # + the deblocking filter
    'cdef': 12,                # + CDEF
    'restoration': 8,          # + superres upscaling and loop restoration, no grain
}


@pytest.mark.parametrize('stage', list(STAGES))
def test_streams_stage_by_stage(av1b, dec, oracle, stage):
    """Every stream with the in-loop stages after `stage` taken out of its
    frames, through the CUDA path and the oracle: the pictures must agree
    frame by frame, so a difference is pinned to the first stage that shows
    it (the job-level isolation the reference gets from replaying its plan
    files, here on real streams above the API boundary)."""
    if not NAMES:
        pytest.skip('no stream fixtures (make -C oracle streams)')
    drop = STAGES[stage]
    bad = []
    for name in NAMES:
        fx = sr.Fixture(name)
        strip = {}

        def rewrite(k, p):
            if k not in strip:
                strip[k] = oracle.strip_stages(p, drop)
            return strip[k]

        mine, _ = sr.replay(fx, dec, rewrite=rewrite)
        ref, _ = sr.replay(fx, oracle.RefDecoder(), rewrite=rewrite)
        if mine != ref:
            bad.append((name, [i for i, (a, b) in enumerate(zip(mine, ref)) if a != b][:4]))
    assert not bad, '%s: %s' % (stage, bad)
