"""The device LJ92 tile encoder and the DNG export of decoded frames
against the CPU oracle (the crate's lj92::encode and dng::tile restated):
every tile's stream byte for byte -- random, smooth and extreme images,
strides wider than the image, images smaller than a tile, tile sizes from
16 to 256 -- and whole DNG files equal to the container around the
oracle's tiles (or the oracle's visible samples), for code values and
linear samples. One device tile is also decoded back by the tests'
lossless JPEG decoder."""

import numpy as np
import pytest
import torch

import _oracle as O
import proresraw_rs_b200 as P
from lj92_decode import decode
from proresraw_rs_b200 import dng as D
from proresraw_rs_b200 import synth as S

pytestmark = pytest.mark.gpu


def device(img, h, stride):
    t = torch.from_numpy(img.reshape(h, stride).astype(np.int32)).to(torch.uint16)
    return t.reshape(-1).cuda()


def images():
    rng = np.random.default_rng(5)
    yield "random", 600, 300, 640, rng.integers(0, 65536, 300 * 640, dtype=np.uint16)
    yy, xx = np.mgrid[0:260, 0:512]
    smooth = (2000 + 800 * np.sin(xx / 37.0) * np.cos(yy / 23.0) + rng.normal(0, 6, xx.shape)).astype(np.uint16)
    yield "smooth", 512, 260, 512, smooth.reshape(-1)
    alt = np.where((np.arange(256 * 64) // 2) % 2 == 0, 0, 0x8000).astype(np.uint16)
    yield "extreme", 256, 64, 256, alt
    yield "ones", 34, 20, 34, np.full(34 * 20, 0xFFFF, np.uint16)
    yield "tiny", 2, 2, 2, np.array([1, 2, 3, 4], np.uint16)
    yield "odd", 257, 255, 258, rng.integers(0, 4096, 255 * 258, dtype=np.uint16)


@pytest.mark.parametrize("tile", [16, 256])
def test_device_tiles_match_the_oracle(tile):
    for name, w, h, stride, img in images():
        got = D.lj92_tiles(device(img, h, stride), w, h, stride, tile)
        want = O.lj92_tiles(img, w, h, tile=tile, stride=stride)
        assert len(got) == len(want), name
        for i, (g, o) in enumerate(zip(got, want)):
            assert g == o, (name, tile, i, len(g), len(o))


def test_other_tile_sizes_and_a_round_trip():
    rng = np.random.default_rng(9)
    w, h = 100, 70
    img = rng.integers(0, 1 << 12, w * h, dtype=np.uint16)
    for tile in (2, 34, 64, 128):
        assert D.lj92_tiles(device(img, h, w), w, h, w, tile) == O.lj92_tiles(img, w, h, tile=tile)
    tiles = D.lj92_tiles(device(img, h, w), w, h, w, 64)
    samples, tw, th, c = decode(tiles[3])
    assert (tw * c, th) == (64, 64)
    assert samples == [int(v) for v in O.dng_tile(img, w, h, 64, 64, 64)]


def frame_of(w, h, pattern, seed):
    m = S.mosaic(w, h, pattern, seed=seed, sigma=12.0, white=4095)
    spec = S.Spec(w, h, pattern=pattern, alignment=2, white_level=4095, valid_tiles=True, wb=(1.9, 1.4),
                  crop=(2, 2, 4, 0), color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
    pkt = S.encode(spec, m, qscale=30, qscale_seed=seed)
    return pkt, P.decode_frame(pkt)


@pytest.mark.parametrize("samples", [D.Samples.CODE_VALUES, D.Samples.LINEAR])
@pytest.mark.parametrize("compression", [D.Compression.LOSSLESS_JPEG, D.Compression.NONE])
def test_dng_files_match_the_container_around_the_oracle(samples, compression):
    w, h = 600, 300
    pkt, frame = frame_of(w, h, S.BGGR, 3)
    of = O.decode_frame(pkt)
    stride = of.header.coded_width
    vis = of.samples.reshape(-1, stride)[:h, :w].reshape(-1)
    if samples == D.Samples.LINEAR:
        vis = of.linearize()
    clip = D.ClipInfo(make="Test", fps=(30, 1), orientation=3)
    got = D.write(frame, clip, samples, compression)
    if compression == D.Compression.NONE:
        chunks = [np.ascontiguousarray(vis, dtype="<u2").tobytes()]
    else:
        chunks = O.lj92_tiles(vis, w, h)
    want = D.assemble(frame.header, chunks, clip, samples, compression)
    assert got == want


def test_a_frame_per_pattern():
    for pattern in (S.RGGB, 1, 2, S.BGGR):
        pkt, frame = frame_of(320, 200, pattern, 10 + pattern)
        of = O.decode_frame(pkt)
        vis = of.samples.reshape(-1, of.header.coded_width)[:200, :320].reshape(-1)
        assert D.write(frame) == D.assemble(frame.header, O.lj92_tiles(vis, 320, 200))


def test_write_into_a_buffer():
    pkt, frame = frame_of(300, 200, S.RGGB, 21)
    want = D.write(frame, D.ClipInfo(make="A"))
    pinned = torch.empty(len(want) + 100, dtype=torch.uint8, pin_memory=True)
    n = D.write_into(frame, pinned, D.ClipInfo(make="A"))
    assert n == len(want) and bytes(pinned[:n].numpy()) == want
    small = bytearray(len(want) - 1)
    with pytest.raises(P.Error) as e:
        D.write_into(frame, small, D.ClipInfo(make="A"))
    assert e.value.code == P._lib.ERR_BUFFER
    big = bytearray(len(want))
    assert D.write_into(frame, big, D.ClipInfo(make="A")) == len(want) and bytes(big) == want


def test_device_output_entry_point():
    # prr_lj92_encode: the streams packed in a device buffer with their
    # offsets on the device, as the host variant returns them; a buffer
    # under the worst-case bound is refused before any launch.
    import ctypes as C

    from proresraw_rs_b200 import _lib

    rng = np.random.default_rng(4)
    w, h, t = 520, 300, 256
    img = rng.integers(0, 1 << 14, w * h, dtype=np.uint16)
    dimg = device(img, h, w)
    L = _lib.lib()
    ctx = P.context()
    n = -(-w // t) * -(-h // t)
    cap = n * int(L.prr_lj92_tile_bound(t))
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    offs = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    assert L.prr_lj92_encode(ctx, dimg.data_ptr(), w, h, w, t, out.data_ptr(), cap, offs.data_ptr()) == 0
    torch.cuda.synchronize()
    o = offs.cpu().numpy()
    data = out[: int(o[-1])].cpu().numpy().tobytes()
    got = [data[int(o[i]):int(o[i + 1])] for i in range(n)]
    assert got == O.lj92_tiles(img, w, h, tile=t)
    assert L.prr_lj92_encode(ctx, dimg.data_ptr(), w, h, w, t, out.data_ptr(), cap - 1,
                             offs.data_ptr()) == _lib.ERR_BUFFER
    assert L.prr_lj92_encode(ctx, dimg.data_ptr(), 1, h, w, t, out.data_ptr(), cap,
                             offs.data_ptr()) == _lib.ERR_INVALID


def image_of_differences(diffs, w, h):
    # The image whose prediction differences, in coding order, are `diffs`
    # (each sample less the one two to its left, the one above for a row's
    # first two, 32768 for the first two of the first row; modulo 2^16).
    img = np.zeros((h, w), dtype=np.int64)
    k = 0
    for r in range(h):
        for c in range(w):
            p = img[r, c - 2] if c >= 2 else (img[r - 1, c] if r > 0 else 32768)
            img[r, c] = (p + int(diffs[k])) % 65536
            k += 1
    return img.astype(np.uint16).reshape(-1)


def test_code_lengths_over_16_bits_are_limited_like_the_crate():
    # Category counts 1, 2, 3, 5, 8, ... (Fibonacci) build a Huffman tree 17
    # deep, so the table must go through the 16-bit length limit; the rest
    # of the 128x128 tile goes to the largest category, which keeps the
    # tree a chain.
    rng = np.random.default_rng(17)
    fib = [1, 2]
    while len(fib) < 17:
        fib.append(fib[-1] + fib[-2])
    cats = rng.permutation(17)
    counts = {int(cats[k]): fib[k] for k in range(17)}
    big = int(cats[16])
    counts[big] += 128 * 128 - sum(fib)
    seq = np.concatenate([np.full(n, c) for c, n in counts.items()])
    rng.shuffle(seq)
    diffs = []
    for c in seq:
        if c == 0:
            diffs.append(0)
        elif c == 16:
            diffs.append(32768)
        else:
            v = int(rng.integers(1 << (c - 1), 1 << c))
            diffs.append(v if rng.random() < 0.5 else -v)
    img = image_of_differences(diffs, 128, 128)
    want = O.lj92_tiles(img, 128, 128, tile=128)
    assert D.lj92_tiles(device(img, 128, 128), 128, 128, 128, 128) == want
    samples, tw, th, c = decode(want[0])
    assert samples == [int(v) for v in O.dng_tile(img, 128, 128, 0, 0, 128)]
