"""A movie of encoded frames through the movie reader and the clip pipeline
(prr_mov_* + prr_clip_*): every frame must be what the oracle's
decode_frame_with / decode_frame_reduced_with gives for that sample's bytes
-- code values or linear RGB bit-exact, the same skipped tiles and
max_qscale, or the same error -- across batch boundaries, for sub-ranges,
with frames of different sizes in one clip, and with a sample that can no
longer be read (the file cut short after it was opened)."""

import os

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import clip as CL
from proresraw_rs_b200 import mov
from proresraw_rs_b200 import synth as S
from proresraw_rs_b200 import synth_movie as M

pytestmark = pytest.mark.gpu

SIZES = ((192, 108), (256, 144), (360, 190), (66, 30))


@pytest.fixture(scope="module")
def packets():
    items = S.mixed_batch(13, seed=5, sizes=SIZES, corrupt=0.02)
    pk = [it.packet for it in items]
    pk[6] = pk[6][:40]  # a packet cut inside its header: the decode reports it
    return pk


@pytest.fixture
def clip_path(tmp_path, packets):
    return M.write_clip(tmp_path / "clip.mov", packets, per_chunk=3, make="Test")


def oracle_of(packet, scale, idct=P.Idct.APPLE, greens=P.Greens.FIRST):
    try:
        if scale is None:
            return O.decode_frame(bytes(packet), int(idct))
        return O.decode_frame_reduced(bytes(packet), int(scale), int(greens))
    except O.OracleError as e:
        return e


def assert_frame(got, want):
    if isinstance(want, O.OracleError):
        assert isinstance(got, P.Error), got
        assert got.code == want.code
        return
    assert not isinstance(got, Exception), got
    assert np.array_equal(got.samples.cpu().numpy().view(np.uint16), want.samples)
    assert got.skipped_tiles == want.skipped_tiles
    assert got.max_qscale == want.max_qscale


@pytest.mark.parametrize("per_batch,threads", [(4, 3), (1, 1), (16, 8)])
def test_every_frame_matches_the_oracle(clip_path, packets, per_batch, threads):
    with mov.read_video_track(clip_path) as track, CL.ClipDecoder(track, per_batch, threads) as dec:
        seen = 0
        for batch in dec.batches():
            assert batch.first == seen
            assert 0 < len(batch.frames) <= per_batch
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], None))
            seen += len(batch.frames)
        assert seen == len(packets)


@pytest.mark.parametrize("scale,greens", [(P.Scale.HALF, P.Greens.FIRST), (P.Scale.QUARTER, P.Greens.AVERAGE)])
def test_reduced_decodes_and_sub_ranges(clip_path, packets, scale, greens):
    with mov.read_video_track(clip_path) as track, CL.ClipDecoder(track, 4, 2) as dec:
        # A full pass, then a sub-range at another scale on the same pipeline.
        assert sum(len(b.frames) for b in dec.batches()) == len(packets)
        firsts = []
        for batch in dec.batches(first=3, count=7, scale=scale, greens=greens):
            firsts.append(batch.first)
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], scale, greens=greens))
        assert firsts == [3, 7]
        # FFmpeg's transform, and an empty range.
        for batch in dec.batches(first=10, idct=P.Idct.FFMPEG):
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], None, P.Idct.FFMPEG))
        assert list(dec.batches(first=5, count=0)) == []


def test_downstream_work_on_the_batch_stream(clip_path, packets):
    # Linearize each frame of each batch before asking for the next: the
    # borrowed outputs are valid until then.
    with mov.read_video_track(clip_path) as track, CL.ClipDecoder(track, 5, 4) as dec:
        for batch in dec.batches():
            for i, got in enumerate(batch.frames):
                want = oracle_of(packets[batch.first + i], None)
                if isinstance(want, O.OracleError):
                    continue
                lin = got.linearize().cpu().numpy().view(np.uint16)
                assert np.array_equal(lin, want.linearize())


def test_a_sample_that_cannot_be_read(tmp_path, packets):
    path = M.write_clip(tmp_path / "cut.mov", packets, per_chunk=3)
    track = mov.read_video_track(path)
    last = track.samples[-1]
    # Cut the file inside the last sample after the track was read (the moov
    # follows the samples, so the table stays as it was read).
    with open(path, "r+b") as f:
        f.truncate(last.offset + last.size // 2)
    seen = 0
    with CL.ClipDecoder(track, 4, 2) as dec:
        # Each batch is checked before the next is asked for: its outputs
        # are borrowed until then.
        for batch in dec.batches():
            for i, got in enumerate(batch.frames):
                k = batch.first + i
                if k == len(packets) - 1:
                    assert isinstance(got, mov.Error)
                    assert str(got) == f"reading {last.size} bytes at byte {last.offset}: failed to fill whole buffer"
                else:
                    assert_frame(got, oracle_of(packets[k], None))
                seen += 1
    assert seen == len(packets)
    track.close()
    os.remove(path)


def test_a_callers_own_sample_table_and_descriptor(clip_path, packets):
    # prr_clip_create_fd: the sample table from another reader (here the
    # library's own, as plain (offset, size) pairs) and a descriptor the
    # caller opened.
    with mov.read_video_track(clip_path) as track:
        samples = [mov.Sample(s.offset, s.size) for s in track.samples]
    fd = os.open(clip_path, os.O_RDONLY)
    try:
        with CL.ClipDecoder.from_fd(fd, samples[2:9], 3, 2) as dec:
            seen = 0
            for batch in dec.batches():
                for i, got in enumerate(batch.frames):
                    assert_frame(got, oracle_of(packets[2 + batch.first + i], None))
                    seen += 1
            assert seen == 7
    finally:
        os.close(fd)


def test_a_queued_range_follows_the_current_one(clip_path, packets):
    # prr_clip_queue: the next range is read and uploaded while the current
    # one drains, then handed out after the current range's end; a queued
    # range may differ in scale and in batch bytes (a sub-range of the
    # smaller frames first, the whole clip queued: the read slots grow).
    small = [i for i, p in enumerate(packets) if len(p) < np.median([len(q) for q in packets])]
    lo = small[0]
    with mov.read_video_track(clip_path) as track, CL.ClipDecoder(track, 3, 2) as dec:
        seen = []
        for k, batch in enumerate(dec.batches(first=lo, count=2)):
            if k == 0:
                dec.queue(scale=P.Scale.HALF, greens=P.Greens.AVERAGE)
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], None))
            seen.append(batch.first)
        assert seen == [lo]
        n = 0
        for batch in dec.queued_batches():
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], P.Scale.HALF, greens=P.Greens.AVERAGE))
            n += len(batch.frames)
        assert n == len(packets)
        # Queued after the current range has ended, and chained again.
        dec.queue(first=4, count=5)
        firsts = []
        for k, batch in enumerate(dec.queued_batches()):
            if k == 0:
                dec.queue(first=0, count=3, idct=P.Idct.FFMPEG)
            firsts.append(batch.first)
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], None))
        assert firsts == [4, 7]
        for batch in dec.queued_batches():
            for i, got in enumerate(batch.frames):
                assert_frame(got, oracle_of(packets[batch.first + i], None, P.Idct.FFMPEG))
        # An empty queued range; a second queued range is refused; a start
        # drops a queued range.
        it = dec.batches(first=0, count=4)
        dec.queue(first=2, count=0)
        with pytest.raises(RuntimeError):
            dec.queue(first=0, count=1)
        assert sum(len(b.frames) for b in it) == 4
        assert list(dec.queued_batches()) == []
        dec.batches(first=0, count=6)
        dec.queue(first=6, count=6)
        assert [b.first for b in dec.batches(first=9, count=4)] == [9, 12]
