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
