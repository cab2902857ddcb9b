"""A movie's frames decoded as a pipeline (prr_clip_* in include/prr.h): the
samples of a `mov.Track` read by host threads into pinned memory and
decoded batch by batch on the device, the reads and uploads of the next
batches overlapping the decode of the current one.

Each frame's result is what `decode_frame_with` (or
`decode_frame_reduced_with`) returns for its sample, or the Error it raises;
a sample that cannot be read gives `mov.Error`::

    with mov.read_video_track(path) as track, ClipDecoder(track) as clip:
        for batch in clip.batches():
            for frame in batch.frames:
                ...  # frame.samples is valid until the next batch
"""

from __future__ import annotations

import ctypes as C
from typing import Iterator, List, Optional, Sequence

from . import Frame, FrameHeader, Greens, Idct, RgbFrame, Scale, _check, _error, _lib, _torch
from . import mov


class _DeviceArray:
    """A borrowed device buffer, for torch.as_tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<u2", "data": (ptr, False), "version": 3,
                                         "strides": None}


class ClipBatch:
    """One decoded batch: `frames[i]` is sample `first + i`'s Frame /
    RgbFrame or Error. Device outputs are borrowed from the pipeline and stay
    valid until the next batch is asked for (`Frame.samples.clone()` keeps
    one)."""

    def __init__(self, first: int, frames: List[object], device_ms: float, busy_ms: float, stream: int):
        self.first = first
        self.frames = frames
        self.device_ms = device_ms  # the batch's kernels, first to last
        self.busy_ms = busy_ms  # of which after the previous batch's kernels ended
        self.stream = stream


class ClipDecoder:
    """The pipeline over an open track: `frames_per_batch` frames a batch,
    `reader_threads` host threads reading samples."""

    def __init__(self, track: Optional[mov.Track], frames_per_batch: int = 8, reader_threads: int = 8,
                 device: Optional[int] = None, _fd: Optional[int] = None, _samples=None):
        torch = _torch()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.track = track  # kept open (and alive) while the pipeline reads it
        h = C.c_void_p()
        if track is not None:
            self._n = len(track.samples)
            rc = _lib.lib().prr_clip_create(self.device, track.handle, frames_per_batch, reader_threads,
                                            C.byref(h))
        else:
            self._n = len(_samples)
            table = (_lib.CMovSample * max(1, self._n))()
            for i, s in enumerate(_samples):
                table[i].offset, table[i].size = int(s.offset), int(s.size)
            rc = _lib.lib().prr_clip_create_fd(self.device, int(_fd), table, self._n, frames_per_batch,
                                               reader_threads, C.byref(h))
        _check(rc)
        self._h = h
        self._ranges: list = []  # (scale, greens) of the current range, then the queued one

    @classmethod
    def from_fd(cls, fd: int, samples: Sequence[mov.Sample], frames_per_batch: int = 8,
                reader_threads: int = 8, device: Optional[int] = None) -> "ClipDecoder":
        """A pipeline over a caller's own sample table and open file
        descriptor (which must stay open), for callers with their own movie
        reader."""
        return cls(None, frames_per_batch, reader_threads, device, _fd=fd, _samples=list(samples))

    def _last_error(self) -> str:
        return _lib.lib().prr_clip_last_error(self._h).decode("utf-8", "replace")

    def batches(self, first: int = 0, count: Optional[int] = None, scale: Optional[Scale] = None,
                idct: Idct = Idct.APPLE, greens: Greens = Greens.FIRST) -> Iterator[ClipBatch]:
        """Decode samples [first, first + count) (count None: to the end) at
        full resolution (scale None, with `idct`) or reduced."""
        L = _lib.lib()
        if count is None:
            count = self._n - first
        sc = _lib.SCALE_FULL if scale is None else int(scale)
        rc = L.prr_clip_start(self._h, first, count, sc, int(idct), int(greens))
        if rc != _lib.OK:
            raise RuntimeError(f"prr_clip_start: {rc} {self._last_error()}")
        self._ranges = [(scale, greens)]
        return self._iterate()

    def queue(self, first: int = 0, count: Optional[int] = None, scale: Optional[Scale] = None,
              idct: Idct = Idct.APPLE, greens: Greens = Greens.FIRST) -> None:
        """prr_clip_queue: the range to decode after the current one; its
        first batches are read and uploaded while the current range drains.
        Iterate it with queued_batches() once the current range has ended."""
        if count is None:
            count = self._n - first
        sc = _lib.SCALE_FULL if scale is None else int(scale)
        rc = _lib.lib().prr_clip_queue(self._h, first, count, sc, int(idct), int(greens))
        if rc != _lib.OK:
            raise RuntimeError(f"prr_clip_queue: {rc} {self._last_error()}")
        self._ranges.append((scale, greens))

    def queued_batches(self) -> Iterator[ClipBatch]:
        """The batches of the range queued with queue(), after the current
        range's batches have all been taken."""
        if len(getattr(self, "_ranges", [])) < 2:
            raise RuntimeError("no range queued")
        self._ranges.pop(0)
        return self._iterate()

    def _iterate(self) -> Iterator[ClipBatch]:
        torch = _torch()
        L = _lib.lib()
        scale, greens = self._ranges[0]
        dev = torch.device("cuda", self.device)
        while True:
            b = _lib.CClipBatch()
            rc = L.prr_clip_next(self._h, C.byref(b))
            if rc != _lib.OK:
                raise RuntimeError(f"prr_clip_next: {rc} {self._last_error()}")
            if b.n == 0:
                return
            frames: List[object] = []
            for i in range(b.n):
                j = b.jobs[i]
                if j.status == _lib.ERR_MOVIE:
                    frames.append(mov.Error(self._last_error()))
                    continue
                if j.status:
                    frames.append(_error(j.status, j.error))
                    continue
                out = torch.as_tensor(_DeviceArray(int(j.dev_out), int(j.out_len)), device=dev)
                header = FrameHeader._from_c(j.result.header)
                n_sk = min(int(j.result.n_skipped), int(j.result.skipped_cap))
                sk = [int(j.result.skipped[k]) for k in range(n_sk)]
                if scale is None:
                    frames.append(Frame(header, out, sk, int(j.result.max_qscale)))
                else:
                    frames.append(RgbFrame(header, scale, greens, out, sk, int(j.result.max_qscale)))
            yield ClipBatch(int(b.first), frames, float(b.device_ms), float(b.busy_ms), int(b.cuda_stream or 0))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().prr_clip_destroy(self._h)
            self._h = None

    def __enter__(self) -> "ClipDecoder":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
