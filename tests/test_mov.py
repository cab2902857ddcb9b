"""The movie reader (libprr.so's host C++ restatement of src/mov.rs) on
hand-built movies: the crate's own tests (src/mov.rs:781-1344), run through
the C ABI, plus exact messages and the corners of the format the crate's
code handles (64-bit atom sizes, version-1 edit lists, rates, lossy UTF-8).
CPU only: no device is touched."""

import os
import struct

import pytest

from proresraw_rs_b200 import mov
from proresraw_rs_b200 import synth_movie as M
from proresraw_rs_b200.synth_movie import ONE, Spec


def prores_raw(fourcc: bytes) -> bool:
    return fourcc in (b"aprn", b"aprh")


def read(path, accept=prores_raw) -> mov.Track:
    return mov.read_video_track(path, accept)


def message(path, accept=prores_raw) -> str:
    with pytest.raises(mov.Error) as e:
        read(path, accept)
    return str(e.value)


def assert_samples(track: mov.Track, first: int, sizes):
    assert len(track.samples) == len(sizes)
    for i, (sample, size) in enumerate(zip(track.samples, sizes)):
        assert sample.size == size
        data = bytearray(size)
        mov.read_at(track, sample.offset, data)
        assert bytes(data) == M.payload(first + i, size), f"sample {i}"


@pytest.fixture
def movie(tmp_path):
    def make(tracks, creation=0, meta=None, name="hand.mov"):
        return M.write_movie(tmp_path / name, tracks, creation, meta)

    return make


def test_chunks_of_several_samples_resolve_after_wide(movie):
    spec = Spec()
    track = read(movie([spec], creation=3_000_000_000))
    assert track.fourcc == b"aprh"
    assert track.fps == (30, 1)
    assert not track.variable_durations
    assert track.creation_time == 3_000_000_000
    assert_samples(track, 0, spec.sizes)


def test_stco_and_co64_agree(movie):
    a = read(movie([Spec()], name="a.mov"))
    b = read(movie([Spec(co64=True)], name="b.mov"))
    assert a == b


@pytest.mark.parametrize("bits", [4, 8, 16])
def test_compact_sizes_of_every_field_width(movie, bits):
    spec = Spec(size_table="stz2", stz2_bits=bits)
    assert_samples(read(movie([spec])), 0, spec.sizes)


def test_edit_list_skips_samples_before_the_first_edit(movie):
    # Media time 15 falls inside sample 0: it starts before the edit, so it
    # is not presented.
    spec = Spec(edits=[(80, 15)])
    track = read(movie([spec], name="a.mov"))
    assert track.warnings == []
    assert_samples(track, 1, spec.sizes[1:])
    # The edit's end bounds the samples too: 20 units from 20 is sample 1 only.
    spec = Spec(edits=[(20, 20)])
    assert_samples(read(movie([spec], name="b.mov")), 1, spec.sizes[1:2])


def test_odd_edit_lists_use_the_first_non_empty_edit_and_warn(movie):
    spec = Spec(edits=[(40, -1), (40, 40), (20, 0)])
    track = read(movie([spec], name="a.mov"))
    assert_samples(track, 2, spec.sizes[2:4])
    assert track.warnings == [
        "the video track's edit list has 3 edits; only the first that shows media is honoured",
        "the video track's edit list starts with an empty edit (a delay), which is ignored",
    ]
    path = movie([Spec(edits=[(20, 1000)])], name="b.mov")
    assert message(path) == "the video track's edit list presents none of its 5 samples"


def test_the_most_common_duration_sets_the_rate(movie):
    # 20 units at 600 per second with an occasional 21; the last sample's
    # odd duration does not count.
    track = read(movie([Spec(durations=[20, 20, 21, 20, 7])], name="a.mov"))
    assert track.fps == (30, 1)
    assert track.variable_durations
    assert not read(movie([Spec(durations=[20, 20, 20, 20, 7])], name="b.mov")).variable_durations


def test_ties_go_to_the_shorter_duration(movie):
    # 21 and 20 twice each (the last sample ignored): 600/20 = 30.
    track = read(movie([Spec(durations=[21, 20, 21, 20, 99])]))
    assert track.fps == (30, 1) and track.variable_durations
    # 24000/1001: the rate is reduced by the gcd.
    track = read(movie([Spec(timescale=24000, durations=[1001] * 5)], name="b.mov"))
    assert track.fps == (24000, 1001)


def test_other_tracks_and_disabled_video_are_skipped(movie):
    sound = Spec(handler=b"soun", fourcc=b"lpcm")
    timecode = Spec(handler=b"tmcd", fourcc=b"tmcd")
    disabled = Spec(enabled=False, fourcc=b"aprn")
    video = Spec(sizes=[9, 8, 7, 6, 5])
    track = read(movie([sound, timecode, disabled, video], name="a.mov"))
    assert track.fourcc == b"aprh"
    assert [s.size for s in track.samples] == video.sizes
    assert_samples(track, 0, video.sizes)
    assert message(movie([sound], name="b.mov")) == "the movie has no enabled video track"


O = mov.Orientation


@pytest.mark.parametrize("matrix,orientation", [
    ((ONE, 0, 0, ONE), O.IDENTITY),
    ((-ONE, 0, 0, ONE), O.MIRROR_HORIZONTAL),
    ((-ONE, 0, 0, -ONE), O.ROTATE_180),
    ((ONE, 0, 0, -ONE), O.MIRROR_VERTICAL),
    ((0, ONE, ONE, 0), O.TRANSPOSE),
    # A phone held upright: the stored frame turns a quarter clockwise.
    ((0, ONE, -ONE, 0), O.ROTATE_90),
    ((0, -ONE, -ONE, 0), O.TRANSVERSE),
    ((0, -ONE, ONE, 0), O.ROTATE_270),
    # Scale is ignored.
    ((-2 * ONE, 0, 0, -ONE // 2), O.ROTATE_180),
])
@pytest.mark.parametrize("tkhd_version", [0, 1])
def test_display_matrices_set_the_orientation(movie, matrix, orientation, tkhd_version):
    track = read(movie([Spec(matrix=matrix, tkhd_version=tkhd_version)]))
    assert track.orientation == orientation
    assert track.warnings == []


def test_orientations_have_their_exif_values():
    order = [O.IDENTITY, O.MIRROR_HORIZONTAL, O.ROTATE_180, O.MIRROR_VERTICAL, O.TRANSPOSE, O.ROTATE_90,
             O.TRANSVERSE, O.ROTATE_270]
    for i, o in enumerate(order):
        assert o.exif() == i + 1
        assert o.swaps_dimensions() == (i >= 4)


def test_other_display_matrices_show_frames_as_stored(movie):
    # 45 degrees.
    track = read(movie([Spec(matrix=(46341, 46341, -46341, 46341))]))
    assert track.orientation == O.IDENTITY
    assert track.warnings == [
        "the video track's display matrix [0.7071075439453125 0.7071075439453125; -0.7071075439453125 "
        "0.7071075439453125] is not a quarter turn or mirror, so the frames are shown as stored"
    ]


def test_other_codecs_are_named(movie):
    path = movie([Spec(fourcc=b"apch")])
    assert message(path) == "the video track is `apch`, not a format this reader accepts"
    # A fourcc that is not printable ASCII is escaped as the crate escapes it.
    path = movie([Spec(fourcc=b"a\x01\xff'")], name="b.mov")
    assert message(path) == "the video track is `a\\x01\\xff\\'`, not a format this reader accepts"


def test_the_default_filter_is_is_prores_raw_fourcc(movie):
    # No filter: aprn / aprh in any case (src/lib.rs:72-75); the crate's
    # test filter is case-sensitive.
    path = movie([Spec(fourcc=b"APRH")])
    assert mov.read_video_track(path).fourcc == b"APRH"
    assert "the video track is `APRH`" in message(path)
    # Any filter: the first accepted track wins, the others are skipped.
    path = movie([Spec(fourcc=b"apch"), Spec(fourcc=b"aprn", sizes=[1, 2, 3, 4, 5])], name="b.mov")
    assert read(path, lambda f: f == b"apch").fourcc == b"apch"
    assert read(path).fourcc == b"aprn"

    # An exception in the filter reaches the caller.
    def boom(f):
        raise KeyError(f)

    with pytest.raises(KeyError):
        read(path, boom)


def test_broken_files_are_described(tmp_path):
    path = tmp_path / "hand.mov"
    data = M.movie_bytes([Spec()])
    # Cut inside the moov: the moov atom claims more than the file holds.
    path.write_bytes(data[:-10])
    text = message(path)
    assert "truncated `moov`" in text
    moov_at = data.rfind(b"moov") - 4
    assert text == (f"truncated `moov` atom at byte {moov_at}: it claims {len(data) - moov_at} bytes and the "
                    f"file has {len(data) - 10 - moov_at} left (an interrupted recording?)")
    # A moov whose child claims more than the moov holds.
    inner = bytearray(data)
    stsz = inner.find(b"stsz") - 4
    inner[stsz:stsz + 4] = struct.pack(">I", 1000)
    path.write_bytes(bytes(inner))
    text = message(path)
    assert text.startswith("truncated `stsz` atom: it claims 1000 bytes and ")
    # No moov at all: the recording stopped before writing it.
    path.write_bytes(data[:moov_at])
    assert message(path) == ("the movie has no `moov` atom, so its frames cannot be found "
                             "(an interrupted recording?)")
    # A sample beyond the end of the file.
    beyond = bytearray(data)
    stco = beyond.find(b"stco") + 12
    beyond[stco:stco + 4] = struct.pack(">I", len(data))
    path.write_bytes(bytes(beyond))
    assert message(path) == (f"sample 0 (bytes {len(data)}..{len(data) + 3}) lies beyond the end of the file "
                             f"at {len(data)} bytes (a truncated file?)")
    path.write_bytes(b"\x89PNG\r\n\x1a\n\0\0\0\rIHDR")
    assert message(path) == "not a QuickTime movie: it starts with `\\r\\n\\x1a\\n`, not `ftyp` or `moov`"
    path.write_bytes(b"")
    assert message(path) == "not a QuickTime movie: the file is empty"


def test_sample_table_disagreements_are_described(movie):
    # stts times 4 samples, stsz sizes 5.
    spec = Spec()
    data = bytearray(M.movie_bytes([spec]))
    stts = data.find(b"stts") + 12  # size, kind, version/flags, entry count -> first run's count
    data[stts:stts + 4] = struct.pack(">I", 4)
    p = movie([spec])
    open(p, "wb").write(bytes(data))
    assert message(p) == ("the video track's sample table disagrees: `stts` times 4 samples, the sizes list 5")
    # Chunks that hold fewer samples than are sized.
    p = movie([Spec(chunks=[2, 2])], name="b.mov")
    assert message(p) == ("the video track's sample table disagrees: its chunks hold 4 of the 5 samples it sizes")
    # Chunks that hold more.
    p = movie([Spec(chunks=[2, 2, 2])], name="c.mov")
    assert message(p) == ("the video track's sample table disagrees: its chunks hold more than the 5 samples "
                          "it sizes")
    p = movie([Spec(durations=[20, 0, 20, 20, 20])], name="d.mov")
    assert message(p) == "the video track has a sample of duration 0"
    p = movie([Spec(timescale=0)], name="e.mov")
    assert message(p) == "the video track's timescale is 0"
    p = movie([Spec(size_table="stz2", stz2_bits=12)], name="f.mov")
    assert message(p) == "`stz2` field size 12 is not 4, 8 or 16 bits"


def test_edit_list_corners(movie):
    # Version 0 edits of rate 2 and an edit that shows no media.
    spec = Spec()
    data = bytearray(M.movie_bytes([Spec(edits=[(40, 20)])]))
    elst = data.find(b"elst") + 4 + 4 + 4  # kind, version/flags, count -> first entry
    data[elst + 8:elst + 12] = struct.pack(">i", 2 * ONE)
    p = movie([spec])
    open(p, "wb").write(bytes(data))
    track = read(p)
    assert track.warnings == ["the video track's edit plays at rate 2; frames are read at normal speed"]
    assert_samples(track, 1, spec.sizes[1:3])
    track = read(movie([Spec(edits=[(40, -1)])], name="b.mov"))
    assert track.warnings == [
        "the video track's edit list starts with an empty edit (a delay), which is ignored",
        "the video track's edit list shows no media; every sample is presented",
    ]
    assert_samples(track, 0, spec.sizes)
    # Duration 0: to the end of the media.
    track = read(movie([Spec(edits=[(0, 40)])], name="c.mov"))
    assert_samples(track, 2, spec.sizes[2:])


def test_version_1_edit_lists_and_64_bit_atom_sizes(tmp_path):
    # A version-1 elst (64-bit duration and time), inside an edts whose
    # header uses the 64-bit size form.
    spec = Spec(edits=[(20, 20)])
    data = M.movie_bytes([spec])
    old_edts = M.atom(b"edts", M.atom(b"elst", M.words([0, 1, 20, 20, ONE])))
    assert old_edts in data
    elst1 = M.full(b"elst", 1, 0, M.words([1]) + struct.pack(">QqI", 20, 20, ONE))
    new_edts = struct.pack(">I", 1) + b"edts" + struct.pack(">Q", 16 + len(elst1)) + elst1
    grow = len(new_edts) - len(old_edts)
    out = bytearray(data.replace(old_edts, new_edts))
    # Grow the enclosing trak and moov sizes.
    for kind in (b"trak", b"moov"):
        at = out.find(kind) - 4
        out[at:at + 4] = struct.pack(">I", struct.unpack(">I", out[at:at + 4])[0] + grow)
    path = tmp_path / "v1.mov"
    path.write_bytes(bytes(out))
    track = read(path)
    assert_samples(track, 1, spec.sizes[1:2])


def test_text_metadata_in_both_meta_forms(movie):
    items = [("com.apple.quicktime.make", "Apple"), ("com.example.table", b"\x01\x02\x03")]
    expected = [("com.apple.quicktime.make", "Apple")]
    for iso in (False, True):
        track = read(movie([Spec()], meta=M.meta_atom(items, iso=iso), name=f"m{iso}.mov"))
        assert track.metadata == expected
        assert track.warnings == []
        assert track.text(["com.apple.proapps.manufacturer", "com.apple.quicktime.make"]) == "Apple"
        assert track.text(["nothing"]) is None


def test_text_metadata_is_lossy_utf8_and_trims_nuls(movie):
    # Invalid UTF-8 sequences become U+FFFD, one per maximal ill-formed
    # subsequence (as String::from_utf8_lossy); trailing NULs are trimmed.
    bad = b"a\xe2\x82b\xf0\x80\x80z\xed\xa0\x80\xc3\xa9\xff\x00\x00"
    track = read(movie([Spec()], meta=M.meta_atom([("k\u00ff", (1, bad))])))
    want = bad.decode("utf-8", "replace").rstrip("\0")
    assert want == "a\ufffdb\ufffd\ufffd\ufffdz\ufffd\ufffd\ufffd\u00e9\ufffd"
    assert track.metadata == [("k\u00ff", want)]


def test_damaged_metadata_costs_the_tags_not_the_frames(movie):
    # A keys atom claiming more entries than it holds.
    meta = bytearray(M.meta_atom([("k", "v")]))
    keys = meta.find(b"keys") + 8
    meta[keys:keys + 4] = struct.pack(">I", 3)
    track = read(movie([Spec()], meta=bytes(meta)))
    assert track.metadata == []
    assert track.warnings == ["the movie's metadata is unreadable: truncated `keys` atom"]
    assert len(track.samples) == 5


def test_reads_past_the_end_name_the_range(movie):
    path = movie([Spec()])
    end = os.path.getsize(path)
    track = read(path)
    buf = bytearray(8)
    with pytest.raises(mov.Error) as e:
        mov.read_at(track, end - 4, buf)
    assert str(e.value) == f"reading 8 bytes at byte {end - 4}: failed to fill whole buffer"
    track.close()
    with pytest.raises(ValueError):
        track.sample(0)


def test_missing_files_are_os_errors(tmp_path):
    with pytest.raises(mov.Error) as e:
        read(tmp_path / "none.mov")
    assert str(e.value) == "No such file or directory (os error 2)"


def test_clips_of_frame_packets(tmp_path):
    # The clip writer used by the clip benchmark: the packets come back.
    packets = [bytes([i]) * (100 + 7 * i) for i in range(11)]
    path = M.write_clip(tmp_path / "clip.mov", packets, make="Test Camera")
    with mov.read_video_track(path) as track:
        assert track.fps == (30, 1)
        assert track.text(["com.apple.quicktime.make"]) == "Test Camera"
        assert [track.sample(i) for i in range(len(packets))] == packets
        assert list(track.sizes) == [len(p) for p in packets]


def test_footage_clips():
    # The sample clips under PRORES_RAW_FOOTAGE (none ship with this
    # repository): each first and last sample is a frame (its size, `prrf`).
    root = os.environ.get("PRORES_RAW_FOOTAGE")
    if not root:
        pytest.skip("PRORES_RAW_FOOTAGE is not set")
    clips = [
        ("sony-fx6-prores_raw/FILMPLUS-ProResRaw-NinjaV-FX6-3.MOV", b"aprn", 708, (50, 1), False, "Sony"),
        ("lumix-s5-prores_raw/a7s III ProRes RAW HQ.mov", b"aprh", 346, (24000, 1001), False, "Sony"),
        ("iphone17-prores_raw/04_A001_09210311_C010.mov", b"aprh", 712, (30, 1), True, "Apple Inc."),
    ]
    for clip, fourcc, frames, fps, variable, make in clips:
        path = os.path.join(root, clip)
        if not os.path.isfile(path):
            continue
        with read(path) as t:
            assert (t.fourcc, len(t.samples), t.fps, t.variable_durations) == (fourcc, frames, fps, variable)
            assert t.creation_time is not None and t.warnings == []
            assert t.text(["com.apple.proapps.manufacturer", "com.apple.quicktime.make"]) == make
            assert t.orientation == O.IDENTITY
            for s in (t.samples[0], t.samples[-1]):
                head = bytearray(8)
                mov.read_at(t, s.offset, head)
                assert struct.unpack(">I", head[:4])[0] == s.size and head[4:] == b"prrf"
    path = os.path.join(root, "iphone17-prores_raw/01_A001_09211049_C068.mov")
    if os.path.isfile(path):
        assert read(path).orientation == O.ROTATE_180


def test_corrupted_movies_fail_cleanly(tmp_path):
    # Random byte changes, truncations and size-field rewrites of valid
    # movies (with metadata, edit lists, both offset widths): every read
    # either succeeds or raises the crate's error, never crashes.
    import random

    rng = random.Random(12)
    bases = [
        M.movie_bytes([Spec(edits=[(40, -1), (40, 40)], co64=True)], creation=5,
                      meta=M.meta_atom([("a", "b"), ("c", b"\x00\x01")])),
        M.movie_bytes([Spec(size_table="stz2", stz2_bits=4), Spec(handler=b"soun")]),
        M.movie_bytes([Spec(tkhd_version=1, matrix=(0, ONE, -ONE, 0))], meta=M.meta_atom([("k", "v")], iso=True)),
    ]
    path = tmp_path / "fuzz.mov"
    outcomes = {"ok": 0, "error": 0}
    for trial in range(600):
        data = bytearray(rng.choice(bases))
        kind = rng.randrange(4)
        if kind == 0:  # random bytes
            for _ in range(rng.randrange(1, 8)):
                data[rng.randrange(len(data))] = rng.randrange(256)
        elif kind == 1:  # truncation
            del data[rng.randrange(1, len(data)):]
        elif kind == 2:  # a 32-bit field set to an extreme
            at = rng.randrange(0, len(data) - 4)
            data[at:at + 4] = struct.pack(">I", rng.choice([0, 1, 2, 7, 8, 0x7FFFFFFF, 0xFFFFFFFF, len(data)]))
        else:  # an atom's size field grown or shrunk
            at = data.find(rng.choice([b"trak", b"stbl", b"stsz", b"stsc", b"meta", b"keys", b"elst", b"tkhd"]))
            if at >= 4:
                size = struct.unpack(">I", data[at - 4:at])[0]
                data[at - 4:at] = struct.pack(">I", max(0, size + rng.choice([-9, -1, 1, 9, 1000])) & 0xFFFFFFFF)
        path.write_bytes(bytes(data))
        try:
            with read(path) as t:
                for s in t.samples[:3]:
                    buf = bytearray(s.size)
                    mov.read_at(t, s.offset, buf)
            outcomes["ok"] += 1
        except mov.Error:
            outcomes["error"] += 1
    assert outcomes["ok"] > 0 and outcomes["error"] > 0, outcomes
