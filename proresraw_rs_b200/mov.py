"""The sample table of one video track of a QuickTime (or ISO base media)
movie, mirroring the crate's `mov` module (src/mov.rs): `read_video_track`,
`read_at`, `Track`, `Sample`, `Orientation`.

The parsing runs in libprr.so (host C++); only the `moov` atom is read into
memory. An open `Track` keeps its file open, so its samples can be read with
positional reads from any number of threads::

    from proresraw_rs_b200 import mov, decode_frame
    with mov.read_video_track("A001_C010.mov") as track:
        packet = track.sample(0)
        frame = decode_frame(packet)
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import os
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib


class Error(Exception):
    """Why a movie could not be read (mov::Error, src/mov.rs:22-42): the
    crate's message, naming the atom or structure at fault."""


class Orientation(enum.IntEnum):
    """How a track's stored frames are turned or mirrored for display
    (src/mov.rs:126-148); the values are the EXIF orientations."""

    IDENTITY = 1
    MIRROR_HORIZONTAL = 2
    ROTATE_180 = 3
    MIRROR_VERTICAL = 4
    TRANSPOSE = 5
    ROTATE_90 = 6
    TRANSVERSE = 7
    ROTATE_270 = 8

    def exif(self) -> int:
        """The EXIF / TIFF `Orientation` value, 1 to 8 (src/mov.rs:150-153)."""
        return int(self)

    def swaps_dimensions(self) -> bool:
        """Whether display swaps the stored width and height (src/mov.rs:154-157)."""
        return int(self) >= 5


@dataclasses.dataclass(frozen=True)
class Sample:
    """Where one sample's bytes are in the file (src/mov.rs:91-98)."""

    offset: int
    size: int


_MSG = 1024


def _prores_raw(fourcc: bytes) -> bool:
    from . import is_prores_raw_fourcc

    return is_prores_raw_fourcc(fourcc)


@dataclasses.dataclass(eq=False)
class Track:
    """One video track of a movie (src/mov.rs:100-124): its format, rate,
    samples and the movie's metadata. Equality compares these fields, as the
    crate's derived `PartialEq` does; the open file is not part of it."""

    fourcc: bytes
    fps: Tuple[int, int]
    variable_durations: bool
    samples: List[Sample]
    creation_time: Optional[int]
    orientation: Orientation
    warnings: List[str]
    metadata: List[Tuple[str, str]]
    _handle: Optional[C.c_void_p] = dataclasses.field(default=None, repr=False)
    _offsets: Optional[np.ndarray] = dataclasses.field(default=None, repr=False)
    _sizes: Optional[np.ndarray] = dataclasses.field(default=None, repr=False)

    def _fields(self):
        return (self.fourcc, self.fps, self.variable_durations, self.samples, self.creation_time,
                self.orientation, self.warnings, self.metadata)

    def __eq__(self, other) -> bool:
        return isinstance(other, Track) and self._fields() == other._fields()

    def text(self, keys: Sequence[str]) -> Optional[str]:
        """The first text metadata value stored under any of `keys`, in that
        order (src/mov.rs:160-169)."""
        for key in keys:
            for k, v in self.metadata:
                if k == key:
                    return v
        return None

    # The open file.

    @property
    def handle(self) -> C.c_void_p:
        if self._handle is None:
            raise ValueError("the track's file is closed")
        return self._handle

    def read_at(self, offset: int, buf) -> None:
        """Positional read of len(buf) bytes at `offset` (mov::read_at,
        src/mov.rs:179-183) into a writable buffer (bytearray, numpy array,
        pinned host tensor's numpy view)."""
        mv = memoryview(buf).cast("B")
        n = mv.nbytes
        msg = C.create_string_buffer(_MSG)
        ptr = C.addressof((C.c_uint8 * max(n, 1)).from_buffer(mv)) if n else None
        rc = _lib.lib().prr_mov_read_at(self.handle, offset, ptr, n, msg, _MSG)
        if rc != _lib.OK:
            raise Error(msg.value.decode("utf-8", "replace"))

    def sample(self, i: int) -> bytes:
        """The bytes of presented sample `i` (a frame packet)."""
        s = self.samples[i]
        buf = bytearray(s.size)
        self.read_at(s.offset, buf)
        return bytes(buf)

    @property
    def offsets(self) -> np.ndarray:
        """Every sample's byte offset, u64."""
        return self._offsets

    @property
    def sizes(self) -> np.ndarray:
        """Every sample's size, u32."""
        return self._sizes

    def close(self) -> None:
        if self._handle is not None:
            _lib.lib().prr_mov_close(self._handle)
            self._handle = None

    def __enter__(self) -> "Track":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_video_track(path, accept: Optional[Callable[[bytes], bool]] = None) -> Track:
    """The first enabled video track whose sample description `accept`s,
    with its samples (mov::read_video_track, src/mov.rs:172-177). `accept`
    defaults to `is_prores_raw_fourcc`; raises `Error` with the crate's
    message."""
    L = _lib.lib()
    raised: List[BaseException] = []

    def trampoline(fourcc_ptr, _user) -> int:
        try:
            fourcc = bytes(fourcc_ptr[i] for i in range(4))
            return 1 if (accept or _prores_raw)(fourcc) else 0
        except BaseException as e:  # re-raised after the call
            raised.append(e)
            return 0

    cb = _lib.MOV_ACCEPT_FN(trampoline)
    handle = C.c_void_p()
    msg = C.create_string_buffer(_MSG)
    rc = L.prr_mov_open(os.fsencode(os.fspath(path)), cb, None, C.byref(handle), msg, _MSG)
    if raised:
        if rc == _lib.OK:
            L.prr_mov_close(handle)
        raise raised[0]
    if rc != _lib.OK:
        if rc == _lib.ERR_MOVIE:
            raise Error(msg.value.decode("utf-8", "replace"))
        raise RuntimeError(f"prr_mov_open: status {rc}")
    try:
        info = _lib.CMovInfo()
        if L.prr_mov_get_info(handle, C.byref(info)) != _lib.OK:
            raise RuntimeError("prr_mov_get_info failed")
        n = int(info.n_samples)
        table = (_lib.CMovSample * max(n, 1))()
        if L.prr_mov_get_samples(handle, 0, n, table) != _lib.OK:
            raise RuntimeError("prr_mov_get_samples failed")
        raw = np.frombuffer(table, dtype=np.dtype([("offset", "<u8"), ("size", "<u4"), ("pad", "<u4")]),
                            count=n)
        offsets = raw["offset"].copy()
        sizes = raw["size"].copy()
        warnings = [L.prr_mov_warning(handle, i).decode("utf-8") for i in range(info.n_warnings)]
        metadata = []
        for i in range(info.n_metadata):
            k, v = C.c_char_p(), C.c_char_p()
            if L.prr_mov_metadata(handle, i, C.byref(k), C.byref(v)) != _lib.OK:
                raise RuntimeError("prr_mov_metadata failed")
            metadata.append((k.value.decode("utf-8"), v.value.decode("utf-8")))
    except BaseException:
        L.prr_mov_close(handle)
        raise
    return Track(
        fourcc=bytes(info.fourcc),
        fps=(int(info.fps_num), int(info.fps_den)),
        variable_durations=bool(info.variable_durations),
        samples=[Sample(int(o), int(s)) for o, s in zip(offsets, sizes)],
        creation_time=int(info.creation_time) if info.has_creation_time else None,
        orientation=Orientation(info.orientation),
        warnings=warnings,
        metadata=metadata,
        _handle=handle,
        _offsets=offsets,
        _sizes=sizes,
    )


def read_at(track: Track, offset: int, buf) -> None:
    """mov::read_at (src/mov.rs:179-183) on the track's open file."""
    track.read_at(offset, buf)
