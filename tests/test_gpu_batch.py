"""The batched decode (prr_batch_*): every job of a mixed batch must give
what the oracle's decode_frame_with / decode_frame_reduced_with gives for
its packet -- code values or linear RGB bit-exact, the same skipped tiles and
max_qscale, or the same error -- whatever the launch shape, with or without
graph replay, and after the autotuner has run."""

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import synth as S

pytestmark = pytest.mark.gpu

SMALL_SIZES = ((192, 108), (256, 144), (360, 190), (512, 270), (66, 30))


def jobs_of(items, idct=P.Idct.APPLE):
    return [P.BatchJob(it.packet, None if it.scale == 0 else P.Scale(it.scale), idct, P.Greens(it.greens))
            for it in items]


def oracle_of(job):
    try:
        if job.scale is None:
            return O.decode_frame(bytes(job.packet), int(job.idct))
        return O.decode_frame_reduced(bytes(job.packet), int(job.scale), int(job.greens))
    except O.OracleError as e:
        return e


def assert_job(job, got, want):
    if isinstance(want, O.OracleError):
        assert isinstance(got, P.Error), got
        assert got.code == want.code
        if want.code in (P._lib.ERR_TILE_OUT_OF_BOUNDS,):
            assert got.fields["tile"] == want.err.index
        return
    assert not isinstance(got, P.Error), got
    host = got.samples_host()
    assert np.array_equal(host, want.samples)
    assert got.skipped_tiles == want.skipped_tiles
    assert got.max_qscale == want.max_qscale


def run_and_check(dec, jobs):
    results = dec.decode(jobs)
    assert len(results) == len(jobs)
    for job, got in zip(jobs, results):
        assert_job(job, got, oracle_of(job))
    return results


@pytest.fixture(scope="module")
def corpus():
    return S.mixed_batch(24, seed=2, sizes=SMALL_SIZES, corrupt=0.02)


def test_mixed_batch_matches_the_oracle(corpus):
    dec = P.BatchDecoder()
    run_and_check(dec, jobs_of(corpus))
    assert dec.last_ms() > 0


def test_mixed_batch_ffmpeg_idct(corpus):
    run_and_check(P.BatchDecoder(), jobs_of(corpus, P.Idct.FFMPEG))


def test_corrupted_frames_keep_their_skipped_lists(corpus):
    jobs = jobs_of(corpus)
    results = P.BatchDecoder().decode(jobs)
    skipped = sum(len(r.skipped_tiles) for r in results)
    assert skipped > 0
    for job, got in zip(jobs, results):
        assert_job(job, got, oracle_of(job))


@pytest.mark.parametrize("stage,per_sm,graph,spt", [(16384, 1, True, 2), (32768, 0, False, 2), (65536, 2, True, 2),
                                                    (98304, 1, True, 2), (16384, 0, True, 1), (32768, 3, True, 1),
                                                    (32768, 0, True, 4), (98304, 2, False, 4)])
def test_every_launch_shape_gives_the_same_frames(corpus, stage, per_sm, graph, spt):
    # Streams per thread of an entropy item (1, 2, 4: items of 64, 128 or
    # 256 tiles) change which CTA decodes which stream and which chunk a
    # segment waits for; every frame stays the oracle's.
    dec = P.BatchDecoder()
    jobs = jobs_of(corpus)
    dec.set_config(dec.bucket(jobs), P.BatchConfig(per_sm, stage, graph, spt))
    run_and_check(dec, jobs)


def test_a_launch_shape_with_other_streams_per_thread_is_refused():
    with pytest.raises(P.Error) as e:
        P.BatchDecoder().set_config(0, P.BatchConfig(0, 32768, True, 3))
    assert e.value.code == P._lib.ERR_INVALID


def test_graph_replay_reads_each_new_batch(corpus):
    # Two batches of one bucket with different contents: the second replay
    # must decode the second batch, not repeat the first.
    dec = P.BatchDecoder()
    a = jobs_of(corpus[:8])
    b = a[::-1]  # same bucket, another frame table
    assert dec.bucket(a) == dec.bucket(b)
    for jobs in (a, b, jobs_of(corpus[8:16]), a):
        run_and_check(dec, jobs)


def test_errors_are_reported_per_job(corpus):
    good = jobs_of(corpus[:4])
    pkt = corpus[0].packet
    truncated = P.BatchJob(pkt[:40])
    bad_tag = P.BatchJob(pkt[:4] + b"xxxx" + pkt[8:])
    # A size table entry reaching past the packet: TileOutOfBounds.
    oob = bytearray(corpus[2].packet)
    table = P.frame_info(bytes(oob)).table_offset
    oob[table] = 0xFF
    oob[table + 1] = 0xFF
    oob_job = P.BatchJob(bytes(oob), None)
    jobs = [good[0], truncated, good[1], bad_tag, oob_job, good[2], good[3]]
    results = P.BatchDecoder().decode(jobs)
    for job, got in zip(jobs, results):
        assert_job(job, got, oracle_of(job))
    assert isinstance(results[1], P.Error) and isinstance(results[3], P.Error)


def test_wrong_output_size_is_a_buffer_error(corpus):
    import torch

    job = jobs_of(corpus[:1])[0]
    out = torch.empty(7, dtype=torch.uint16, device="cuda")
    (res,) = P.BatchDecoder().decode([job], outs=[out])
    assert isinstance(res, P.Error) and res.code == P._lib.ERR_BUFFER


def test_empty_and_all_invalid_batches():
    dec = P.BatchDecoder()
    assert dec.decode([]) == []
    res = dec.decode([P.BatchJob(b"\x00" * 12), P.BatchJob(b"")])
    assert all(isinstance(r, P.Error) for r in res)


def test_autotuner_picks_a_config_and_frames_stay_exact(corpus):
    dec = P.BatchDecoder()
    jobs = jobs_of(corpus[:12])
    cfg, ms = dec.tune(jobs, reps=1)
    assert ms > 0 and cfg.stage_bytes % 16 == 0 and cfg.ctas_per_sm >= 1 and cfg.streams_per_thread in (1, 2, 4)
    assert dec.get_config(dec.bucket(jobs)) == cfg
    run_and_check(dec, jobs)


def test_batch_of_one_large_frame_matches_single_decode():
    items = S.mixed_batch(2, seed=11, sizes=((1920, 1080),), corrupt=0.005)
    run_and_check(P.BatchDecoder(), jobs_of(items))


def test_two_decoders_on_two_streams_pipeline(corpus):
    # submit() returns with the batch queued; a second decoder, made under
    # another stream, stages and submits the next batch before the first is
    # waited for. Every batch still matches the oracle, outputs included
    # after the other decoder has written its own.
    import torch

    jobs_a, jobs_b = jobs_of(corpus[:12]), jobs_of(corpus[12:])
    decs = []
    for _ in range(2):
        with torch.cuda.stream(torch.cuda.Stream()):
            decs.append(P.BatchDecoder())
    assert decs[0].ctx.value != decs[1].ctx.value
    want = {id(j): oracle_of(j) for j in jobs_a + jobs_b}
    order = [jobs_a, jobs_b, jobs_a, jobs_b]
    decs[0].submit(order[0])
    for k in range(1, len(order) + 1):
        if k < len(order):
            decs[k % 2].submit(order[k])
        got = decs[(k - 1) % 2].wait()
        for job, g in zip(order[k - 1], got):
            assert_job(job, g, want[id(job)])


def test_submit_twice_or_wait_without_submit_is_invalid(corpus):
    dec = P.BatchDecoder()
    with pytest.raises(P.Error) as e:
        dec.wait()
    assert e.value.code == P._lib.ERR_INVALID
    jobs = jobs_of(corpus[:4])
    dec.submit(jobs)
    with pytest.raises(P.Error) as e:
        dec.submit(jobs)
    assert e.value.code == P._lib.ERR_INVALID
    for job, g in zip(jobs, dec.wait()):
        assert_job(job, g, oracle_of(job))


def test_a_chunk_that_never_finishes_times_out_and_the_context_stays_usable():
    """A bounded device wait that runs out. The test hook abandons the first
    entropy chunk of the batch, so its flag is never set: the segments of
    the first frame that wait for it give up after the (shortened) limit,
    that frame reports PRR_ERR_TIMEOUT, the other frames are still exact,
    and the next batch on the same context is exact too."""
    import time

    items = S.mixed_batch(6, seed=7, sizes=SMALL_SIZES, corrupt=0.0)
    jobs = jobs_of(items)
    wants = [oracle_of(j) for j in jobs]
    assert not isinstance(wants[0], O.OracleError)
    dec = P.BatchDecoder()
    dec.set_wait_limit(20_000)  # 20 ms
    dec.drop_chunk_for_test(0)
    t0 = time.perf_counter()
    got = dec.decode(jobs)
    elapsed = time.perf_counter() - t0
    assert isinstance(got[0], P.Error) and got[0].code == P._lib.ERR_TIMEOUT, got[0]
    for job, g, w in zip(jobs[1:], got[1:], wants[1:]):
        assert_job(job, g, w)
    assert elapsed < 10.0  # the waits ended after their limit, not after the 2 s default
    dec.drop_chunk_for_test(None)
    dec.set_wait_limit(0)
    for job, g, w in zip(jobs, dec.decode(jobs), wants):
        assert_job(job, g, w)
