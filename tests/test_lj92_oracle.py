"""The CPU oracle of the DNG export's lossless JPEG encoder, pinned by the
reference's own tests of it (examples/prr2dng/lj92.rs:340-399,
examples/prr2dng/dng.rs:238-248): round trips through a decoder, a flat
tile's size, the Huffman table of a skewed histogram, the tile cut's edge
padding. CPU only."""

import numpy as np
import pytest

import _oracle as O
from lj92_decode import decode


def round_trip(samples, width, height):
    data = O.lj92_encode(np.asarray(samples, np.uint16), width, height, 2)
    decoded, w, h, c = decode(data)
    assert (w, h, c) == (width // 2, height, 2)
    assert decoded == [int(v) for v in samples]
    return data


def xorshift(n, state=0x123456789ABCDEF0):
    out = []
    m = (1 << 64) - 1
    for _ in range(n):
        state ^= (state << 13) & m
        state ^= state >> 7
        state ^= (state << 17) & m
        out.append(state & 0xFFFF)
    return out


def test_random_and_extreme_samples_survive():
    round_trip(xorshift(64 * 16), 64, 16)
    # Differences of exactly +-32768 and runs of 0xFF bytes.
    round_trip([0 if (i // 2) % 2 == 0 else 0x8000 for i in range(32 * 4)], 32, 4)
    round_trip([0xFFFF] * (16 * 2), 16, 2)


def test_a_flat_tile_still_gets_a_valid_table():
    data = round_trip([1000] * 256, 16, 16)
    # Smooth data compresses: here to well under a bit per sample.
    assert len(data) < 16 * 16 // 8 + 64, len(data)


def test_skewed_histograms_need_long_codes():
    # Frequencies growing fourfold per category force lengths past 16
    # before limiting.
    counts, values, codes, lengths = O.lj92_huffman([1 << (2 * i) for i in range(17)])
    assert all(1 <= int(l) <= 16 for l in lengths)
    # Kraft: the codes leave room for the reserved all-ones code.
    assert sum(0.5 ** int(l) for l in lengths) < 1.0
    assert not any(int(c) == (1 << int(l)) - 1 for c, l in zip(codes, lengths))
    assert int(counts.sum()) == len(values) == 17


def test_tables_are_canonical_and_prefix_free():
    rng = np.random.default_rng(3)
    for _ in range(50):
        hist = rng.integers(0, 1000, 17) * (rng.random(17) < 0.7)
        hist[int(rng.integers(17))] += 1
        counts, values, codes, lengths = O.lj92_huffman(hist)
        used = [v for v in range(17) if hist[v] > 0]
        assert sorted(int(v) for v in values) == used
        words = [format(int(codes[v]), f"0{int(lengths[v])}b") for v in used]
        for a in words:
            assert a != "1" * len(a)
            for b in words:
                assert a == b or not b.startswith(a)
        # Shorter codes for more frequent categories (before length limits).
        by_len = sorted(used, key=lambda v: int(lengths[v]))
        assert hist[by_len[0]] >= min(hist[v] for v in used)


def test_padding_repeats_the_edge_of_the_same_colour():
    # A 4x2 image whose value is its column plus 10 x its row.
    values = np.array([i % 4 + 10 * (i // 4) for i in range(8)], np.uint16)
    tile = O.dng_tile(values, 4, 2, 0, 0)
    assert list(tile[:8]) == [0, 1, 2, 3, 2, 3, 2, 3]
    assert list(tile[256:260]) == [10, 11, 12, 13]
    # Rows past the bottom alternate between the last two rows.
    assert tile[2 * 256] == 0 and tile[3 * 256] == 10


def test_tiles_of_an_image_cover_it():
    # A 70x36 image: 3x2 tiles of 32, cut and encoded in order; each decodes
    # to its cut, and the cuts reassemble the image.
    w, h, t = 70, 36, 32
    img = np.array(xorshift(w * h, 77), np.uint16) >> 4
    streams = O.lj92_tiles(img, w, h, tile=t, threads=2)
    across, down = -(-w // t), -(-h // t)
    assert len(streams) == across * down
    for i, s in enumerate(streams):
        got, tw, th, c = decode(s)
        assert (tw * c, th) == (t, t)
        cut = O.dng_tile(img, w, h, i % across * t, i // across * t, t)
        assert got == [int(v) for v in cut]
        assert s == O.lj92_encode(cut, t, t)
    # A stride wider than the image reads the same picture.
    wide = np.zeros((h, w + 10), np.uint16)
    wide[:, :w] = img.reshape(h, w)
    assert O.lj92_tiles(wide, w, h, tile=t, stride=w + 10) == streams


@pytest.mark.parametrize("n", [1, 3])
def test_images_smaller_than_a_tile_repeat_their_edges(n):
    w, h = 2 * n, 2
    img = np.arange(w * h, dtype=np.uint16) * 1000
    tile = O.dng_tile(img, w, h, 0, 0, 8)
    for y in range(8):
        for x in range(8):
            cx = x if x < w else w - 2 + (x - w) % 2
            cy = y if y < h else h - 2 + (y - h) % 2
            assert tile[y * 8 + x] == img[cy * w + cx]
