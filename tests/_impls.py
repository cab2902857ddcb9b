"""Two implementations behind one interface, so a test reads like the
crate's own test and runs against the CPU oracle (always) and the CUDA
library (on a GPU).

Every method returns host numpy data so that results compare directly.
"""

from __future__ import annotations

import numpy as np

import _oracle as O


class Decoded:
    def __init__(self, header, samples, skipped, max_qscale):
        self.header = header  # has width, height, coded_width(), bayer_pattern, curve, quant_matrix...
        self.samples = samples
        self.skipped_tiles = list(skipped)
        self.max_qscale = max_qscale

    def width(self):
        return self.header.width

    def height(self):
        return self.header.height

    def stride(self):
        return (self.header.width + 15) & ~15

    def quantizer(self):
        return int(self.header.quant_matrix[0]) * int(self.max_qscale)


class OracleImpl:
    name = "oracle"

    def decode(self, packet, idct=0):
        f = O.decode_frame(packet, idct)
        return Decoded(f.header, f.samples, f.skipped_tiles, f.max_qscale), f

    def decode_reduced(self, packet, shift, greens):
        f = O.decode_frame_reduced(packet, shift, greens)
        return Decoded(f.header, f.samples, f.skipped_tiles, f.max_qscale)

    def linearize(self, raw):
        return raw.linearize()

    def params(self, header, q, red=None, blue=None):
        if red is None:
            return O.params_new(header, q)
        return O.params_with_white_balance(header, q, red, blue)

    def develop(self, raw, params, stage, planar):
        return O.develop(raw, params, stage, planar)


class GpuImpl:
    name = "gpu"

    def __init__(self):
        import proresraw_rs_b200 as P

        self.P = P

    def decode(self, packet, idct=0):
        f = self.P.decode_frame_with(packet, self.P.Idct(idct))
        h = f.header
        return Decoded(_HeaderView(h), f.samples_host(), f.skipped_tiles, f.max_qscale), f

    def decode_reduced(self, packet, shift, greens):
        f = self.P.decode_frame_reduced_with(packet, self.P.Scale(shift), self.P.Greens(greens))
        return Decoded(_HeaderView(f.header), f.samples_host(), f.skipped_tiles, f.max_qscale)

    def linearize(self, raw):
        return raw.linearize().cpu().numpy().view(np.uint16)

    def params(self, header, q, red=None, blue=None):
        if red is None:
            return self.P.DemosaicParams.new(header, q)
        return self.P.DemosaicParams.with_white_balance(header, q, red, blue)

    def develop(self, raw, params, stage, planar):
        P = self.P
        if planar:
            pl = P.develop_planar(raw, params, P.Stage(stage))
            return tuple(t.cpu().numpy() for t in pl.planes)
        img = P.develop_with(raw, params, P.Stage(stage))
        return img.data.cpu().numpy()


class _HeaderView:
    """Oracle-style attribute access to a FrameHeader."""

    def __init__(self, h):
        self._h = h
        self.width, self.height = h.width, h.height
        self.bayer_pattern = int(h.bayer_pattern)
        self.quant_matrix = h.quant_matrix
        self.curve = h.curve.points
        self.white_level = h.white_level
        self.alignment = h.alignment


def header_fields(h):
    """Comparable tuple of header fields for oracle and library headers."""
    if hasattr(h, "_h"):
        h = h._h
    if hasattr(h, "curve") and hasattr(h.curve, "points"):
        m = [v for row in h.color_matrix for v in row]
        return (h.version, bytes(h.vendor), h.width, h.height, tuple(h.crop), int(h.bayer_pattern), h.white_level,
                h.wb_red, h.wb_blue, tuple(m), h.gain, h.wb_cct, h.flags, h.alignment, tuple(h.quant_matrix),
                tuple(h.curve.points))
    return (h.version, bytes(h.vendor), h.width, h.height, tuple(h.crop), int(h.bayer_pattern), h.white_level,
            h.wb_red, h.wb_blue, tuple(h.color_matrix), h.gain, h.wb_cct, h.flags, h.alignment,
            tuple(h.quant_matrix), tuple(h.curve))
