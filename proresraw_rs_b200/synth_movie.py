"""Hand-built QuickTime movies: the atoms a video track's sample table is
read from, written the way the crate's own tests build theirs
(src/mov.rs:810-995), plus clips whose samples are real frame packets.

Used by the tests of the movie reader and by the clip benchmark (a movie of
synthetic frames on local disk, since no camera clip is available).
"""

from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional, Sequence, Tuple

ONE = 0x10000  # 1.0 in 16.16


def atom(kind: bytes, body: bytes) -> bytes:
    return struct.pack(">I", len(body) + 8) + kind + body


def full(kind: bytes, version: int, flags: int, body: bytes) -> bytes:
    """An atom whose body starts with a version byte and 24 flag bits."""
    return atom(kind, struct.pack(">I", flags | version << 24) + body)


def words(values: Sequence[int]) -> bytes:
    return b"".join(struct.pack(">I", v & 0xFFFFFFFF) for v in values)


def payload(i: int, size: int) -> bytes:
    """Sample i's bytes in the hand-built movies: `size` copies of i."""
    return bytes([i & 0xFF]) * size


@dataclasses.dataclass
class Spec:
    """One track. The defaults are the crate's test movie: five samples of
    20 units at 600 per second in chunks of 2, 2 and 1."""

    handler: bytes = b"vide"
    fourcc: bytes = b"aprh"
    enabled: bool = True
    timescale: int = 600
    durations: List[int] = dataclasses.field(default_factory=lambda: [20] * 5)
    sizes: List[int] = dataclasses.field(default_factory=lambda: [3, 5, 7, 2, 4])
    size_table: str = "stsz"  # or "stz2"
    stz2_bits: int = 16
    chunks: List[int] = dataclasses.field(default_factory=lambda: [2, 2, 1])
    co64: bool = False
    edits: List[Tuple[int, int]] = dataclasses.field(default_factory=list)  # (segment duration, media time)
    tkhd_version: int = 0
    matrix: Tuple[int, int, int, int] = (ONE, 0, 0, ONE)  # a b c d, 16.16
    payloads: Optional[List[bytes]] = None  # None: payload(i, size)

    def data(self) -> bytes:
        if self.payloads is not None:
            return b"".join(self.payloads)
        return b"".join(payload(i, s) for i, s in enumerate(self.sizes))


def trak(spec: Spec, data: int) -> bytes:
    """A `trak` whose samples start at byte `data` of the file, back to back."""
    at = 40 if spec.tkhd_version == 0 else 52
    tkhd = bytearray(at + 44)
    tkhd[:4] = struct.pack(">I", int(spec.enabled) | spec.tkhd_version << 24)
    a, b, c, d = spec.matrix
    for i, v in enumerate([a, b, 0, c, d, 0, 0, 0, 0x40000000]):
        tkhd[at + 4 * i:at + 4 * i + 4] = struct.pack(">i", v)
    body = atom(b"tkhd", bytes(tkhd))
    if spec.edits:
        elst = words([0, len(spec.edits)])
        for duration, time in spec.edits:
            elst += words([duration, time, ONE])
        body += atom(b"edts", atom(b"elst", elst))
    entry = bytearray(78)
    entry[7] = 1
    stbl = full(b"stsd", 0, 0, words([1]) + atom(spec.fourcc, bytes(entry)))
    runs: List[List[int]] = []
    for dur in spec.durations:
        if runs and runs[-1][1] == dur:
            runs[-1][0] += 1
        else:
            runs.append([1, dur])
    stbl += full(b"stts", 0, 0, words([len(runs)] + [x for r in runs for x in r]))
    stsc, count = b"", 0
    for i, n in enumerate(spec.chunks):
        if i == 0 or spec.chunks[i - 1] != n:
            stsc += words([i + 1, n, 1])
            count += 1
    stbl += full(b"stsc", 0, 0, words([count]) + stsc)
    n = len(spec.sizes)
    if spec.size_table == "stsz":
        stbl += full(b"stsz", 0, 0, words([0, n] + list(spec.sizes)))
    else:
        bits = spec.stz2_bits
        if bits == 4:
            s = list(spec.sizes) + [0]
            table = bytes((s[k] << 4 | (s[k + 1] if k + 1 < n else 0)) & 0xFF for k in range(0, n, 2))
        elif bits == 8:
            table = bytes(s & 0xFF for s in spec.sizes)
        else:
            table = b"".join(struct.pack(">H", s & 0xFFFF) for s in spec.sizes)
        stbl += full(b"stz2", 0, 0, bytes([0, 0, 0, bits]) + words([n]) + table)
    offsets, pos, k = [], data, 0
    for cn in spec.chunks:
        offsets.append(pos)
        pos += sum(spec.sizes[k:k + cn])
        k += cn
    if spec.co64:
        stbl += full(b"co64", 0, 0, words([len(offsets)]) + b"".join(struct.pack(">Q", o) for o in offsets))
    else:
        stbl += full(b"stco", 0, 0, words([len(offsets)] + offsets))
    minf = full(b"vmhd", 0, 1, bytes(8)) + atom(b"stbl", stbl)
    mdia = full(b"mdhd", 0, 0, words([0, 0, spec.timescale, 0, 0]))
    mdia += full(b"hdlr", 0, 0, b"mhlr" + spec.handler + bytes(13))
    mdia += atom(b"minf", minf)
    body += atom(b"mdia", mdia)
    return atom(b"trak", body)


def meta_atom(items: Sequence[Tuple[str, object]], iso: bool = False) -> bytes:
    """A `meta` atom with `mdta` keys: (key, value) where a str value is
    stored as UTF-8 (type 1), bytes as binary (type 0) and a (type, bytes)
    pair as given. `iso` adds the version and flags word of the ISO form."""
    keys = words([0, len(items)])
    ilst = b""
    for i, (key, value) in enumerate(items):
        k = key.encode("utf-8")
        keys += words([len(k) + 8]) + b"mdta" + k
        if isinstance(value, str):
            kind, raw = 1, value.encode("utf-8")
        elif isinstance(value, tuple):
            kind, raw = value
        else:
            kind, raw = 0, bytes(value)
        ilst += atom(struct.pack(">I", i + 1), atom(b"data", words([kind, 0]) + raw))
    children = full(b"hdlr", 0, 0, b"\0\0\0\0mdta" + bytes(12)) + atom(b"keys", keys) + atom(b"ilst", ilst)
    return atom(b"meta", (bytes(4) if iso else b"") + children)


def movie_bytes(tracks: Sequence[Spec], creation: int = 0, meta: Optional[bytes] = None) -> bytes:
    """ftyp, wide, mdat holding every track's samples in turn, then moov."""
    out = atom(b"ftyp", b"qt  \0\0\x02\0qt  ") + atom(b"wide", b"")
    data, starts = b"", []
    for spec in tracks:
        starts.append(len(out) + 8 + len(data))
        data += spec.data()
    out += atom(b"mdat", data)
    moov = full(b"mvhd", 0, 0, words([creation, 0, 600, 0]))
    for spec, start in zip(tracks, starts):
        moov += trak(spec, start)
    if meta is not None:
        moov += meta
    return out + atom(b"moov", moov)


def write_movie(path, tracks: Sequence[Spec], creation: int = 0, meta: Optional[bytes] = None) -> str:
    with open(path, "wb") as f:
        f.write(movie_bytes(tracks, creation, meta))
    return str(path)


def write_clip(path, packets: Sequence[bytes], fourcc: bytes = b"aprh", timescale: int = 600,
               duration: int = 20, per_chunk: int = 4, make: Optional[str] = None) -> str:
    """A movie whose video track's samples are `packets`, `per_chunk`
    samples to a chunk, with 64-bit chunk offsets when the data passes 4 GiB."""
    n = len(packets)
    chunks = [per_chunk] * (n // per_chunk) + ([n % per_chunk] if n % per_chunk else [])
    spec = Spec(fourcc=fourcc, timescale=timescale, durations=[duration] * n, sizes=[len(p) for p in packets],
                chunks=chunks, co64=sum(len(p) for p in packets) >= 1 << 32, payloads=list(packets))
    meta = meta_atom([("com.apple.quicktime.make", make)]) if make else None
    return write_movie(path, [spec], creation=3_000_000_000, meta=meta)
