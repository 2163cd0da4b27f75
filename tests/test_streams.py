"""The oracle on real streams: the reference's 24 bit-exact test streams, run
through the reference's own front end by oracle/stream_dump into replay
fixtures, replayed through the oracle (the reference CPU backend) from this
repository's serialized FrameSyntax blobs, must reproduce the dav1d frame
hashes the reference's stream tests check (CMakeLists.txt:272-350 of the
reference). This pins the oracle, the blob format and the replay order end
to end; tests/test_streams_gpu.py holds the CUDA path to the same hashes."""
import pytest

import stream_replay as sr

NAMES = sr.fixture_names()
LEVEL_NAMES = sr.fixture_names(levels=True)


def need_fixtures():
    if not NAMES:
        pytest.skip('no stream fixtures (make -C oracle streams)')


def test_all_streams_present():
    need_fixtures()
    assert len(NAMES) == 24, NAMES
    assert LEVEL_NAMES == NAMES


@pytest.mark.parametrize('name', NAMES or ['none'])
def test_oracle_matches_stream_hashes(oracle, name):
    need_fixtures()
    fx = sr.Fixture(name)
    got, _ = sr.replay(fx, oracle.RefDecoder())
    assert len(got) == len(fx.hashes)
    bad = [i for i, (a, b) in enumerate(zip(got, fx.hashes)) if a != b]
    assert not bad, '%s: frames %s differ from the recorded hashes' % (name, bad[:8])


@pytest.mark.parametrize('name', LEVEL_NAMES or ['none'])
def test_levels_fixture_matches_coefficient_fixture(av1b, oracle, name):
    """The device-dequantiser form of a stream carries the same frames as the
    dequantised form, with the coded levels instead of the coefficient pool."""
    need_fixtures()
    a, b = sr.Fixture(name), sr.Fixture(name, levels=True)
    assert a.hashes == b.hashes
    assert [e[:3] for e in a.events] == [e[:3] for e in b.events]
    levels = 0
    for (_, _, _, pa), (_, _, _, pb) in zip(a.decodes(), b.decodes()):
        ba, bb = av1b.Blob.from_bytes(pa), av1b.Blob.from_bytes(pb)
        assert ba.header == bb.header
        ca, cb = oracle.blob_counts(ba), oracle.blob_counts(bb)
        assert cb['coefficients'] == 0
        levels += cb['levels']
        for k in oracle.BLOB_ARRAYS:
            if k not in ('coefficients', 'levels'):
                assert ca[k] == cb[k], k
    assert levels > 0


@pytest.mark.parametrize('name', LEVEL_NAMES or ['none'])
def test_host_expansion_of_levels_matches_stream_hashes(oracle, name):
    """The levels fixtures, expanded on the host by the reference front end's
    own dequantiser (through an identity quantiser matrix on every transform,
    so the matrix path runs too), decode to the dav1d hashes: the levels,
    offsets and steps the device dequantiser reads are pinned."""
    need_fixtures()
    fx = sr.Fixture(name, levels=True)
    got, _ = sr.replay(fx, oracle.RefDecoder(),
                       rewrite=lambda k, p: oracle.dequant_pair(p, 0)[1])
    assert got == fx.hashes
