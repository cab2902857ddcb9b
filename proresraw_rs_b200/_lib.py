"""ctypes declarations of include/prr.h (libprr.so)."""

from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libprr.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "prr.h")

OK = 0
ERR_TRUNCATED = -1
ERR_FRAME_SIZE_MISMATCH = -2
ERR_BAD_QUANT_MATRIX = -3
ERR_BAD_CURVE = -4
ERR_UNEXPECTED_CURVE = -5
ERR_BAD_TAG = -6
ERR_HEADER_TOO_SHORT = -7
ERR_UNSUPPORTED_VERSION = -8
ERR_BAD_DIMENSIONS = -9
ERR_BAD_ALIGNMENT = -10
ERR_TILE_OUT_OF_BOUNDS = -11
ERR_BAD_TILE_HEADER = -12
ERR_BUFFER = -20
ERR_CUDA = -21
ERR_TIMEOUT = -22
ERR_INVALID = -23
ERR_NO_MEMORY = -24
ERR_SCRATCH_LIMIT = -25
ERR_MOVIE = -26
NOALLOC_MAX_TILES = 262144


class CError(C.Structure):
    _fields_ = [
        ("code", C.c_int32),
        ("what", C.c_char * 32),
        ("needed", C.c_uint64),
        ("available", C.c_uint64),
        ("declared", C.c_uint32),
        ("actual", C.c_uint64),
        ("index", C.c_uint64),
        ("value", C.c_uint32),
        ("width", C.c_uint16),
        ("height", C.c_uint16),
        ("curve", C.c_uint16 * 8),
        ("tag", C.c_uint8 * 4),
    ]


class CHeader(C.Structure):
    _fields_ = [
        ("version", C.c_uint8),
        ("vendor", C.c_uint8 * 4),
        ("bayer_pattern", C.c_uint8),
        ("width", C.c_uint16),
        ("height", C.c_uint16),
        ("crop", C.c_uint8 * 4),
        ("white_level", C.c_uint16),
        ("wb_cct", C.c_uint16),
        ("flags", C.c_uint16),
        ("alignment", C.c_uint8),
        ("pad0", C.c_uint8),
        ("wb_red", C.c_float),
        ("wb_blue", C.c_float),
        ("color_matrix", C.c_float * 9),
        ("gain", C.c_float),
        ("quant_matrix", C.c_uint8 * 64),
        ("curve", C.c_uint16 * 8),
    ]


class CFrameInfo(C.Structure):
    _fields_ = [
        ("header", CHeader),
        ("packet_len", C.c_uint64),
        ("table_offset", C.c_uint64),
        ("ntiles", C.c_uint32),
        ("tiles_per_row", C.c_uint32),
        ("tile_rows", C.c_uint32),
        ("coded_width", C.c_uint32),
        ("coded_height", C.c_uint32),
        ("pad0", C.c_uint32),
    ]


class CParams(C.Structure):
    _fields_ = [
        ("cfa_phase", C.c_int32),
        ("black", C.c_int32),
        ("one_over_range", C.c_float),
        ("noise", C.c_float * 3),
        ("clip", C.c_float * 2),
        ("black_over_range", C.c_float),
        ("wb", C.c_float * 2),
    ]


class CDecodeResult(C.Structure):
    _fields_ = [
        ("header", CHeader),
        ("n_skipped", C.c_uint64),
        ("skipped", C.POINTER(C.c_uint64)),
        ("skipped_cap", C.c_uint64),
        ("max_qscale", C.c_uint8),
        ("pad", C.c_uint8 * 7),
    ]


class CDevStatus(C.Structure):
    _fields_ = [
        ("oob_tile", C.c_uint32),
        ("n_skipped", C.c_uint32),
        ("max_qscale", C.c_uint32),
        ("error", C.c_uint32),
    ]


class CJob(C.Structure):
    _fields_ = [
        ("packet", C.c_void_p),
        ("len", C.c_uint64),
        ("scale", C.c_int32),
        ("idct", C.c_int32),
        ("greens", C.c_int32),
        ("status", C.c_int32),
        ("dev_out", C.c_void_p),
        ("out_len", C.c_uint64),
        ("result", CDecodeResult),
        ("error", CError),
    ]


class CDevelopConfig(C.Structure):
    _fields_ = [
        ("tile_w", C.c_uint32),
        ("tile_h", C.c_uint32),
        ("ctas_per_sm", C.c_uint32),
    ]


class CBatchConfig(C.Structure):
    _fields_ = [
        ("ctas_per_sm", C.c_uint32),
        ("stage_bytes", C.c_uint32),
        ("use_graph", C.c_uint32),
        ("streams_per_thread", C.c_uint32),
    ]


class CSgModel(C.Structure):
    _fields_ = [
        ("dev_params", C.c_void_p),
        ("noise_lo", C.c_float),
        ("noise_hi", C.c_float),
    ]


class CMovSample(C.Structure):
    _fields_ = [
        ("offset", C.c_uint64),
        ("size", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class CMovInfo(C.Structure):
    _fields_ = [
        ("fourcc", C.c_uint8 * 4),
        ("fps_num", C.c_uint32),
        ("fps_den", C.c_uint32),
        ("variable_durations", C.c_uint8),
        ("orientation", C.c_uint8),
        ("has_creation_time", C.c_uint8),
        ("reserved", C.c_uint8),
        ("creation_time", C.c_uint64),
        ("n_samples", C.c_uint64),
        ("n_warnings", C.c_uint32),
        ("n_metadata", C.c_uint32),
    ]


MOV_ACCEPT_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_uint8), C.c_void_p)


class CClipBatch(C.Structure):
    _fields_ = [
        ("first", C.c_uint64),
        ("n", C.c_uint32),
        ("device_ms", C.c_float),
        ("busy_ms", C.c_float),
        ("pad", C.c_uint32),
        ("jobs", C.POINTER(CJob)),
        ("cuda_stream", C.c_void_p),
    ]

class CDngClip(C.Structure):
    _fields_ = [
        ("make", C.c_char_p),
        ("model", C.c_char_p),
        ("date_time", C.c_char_p),
        ("software", C.c_char_p),
        ("fps_num", C.c_uint32),
        ("fps_den", C.c_uint32),
        ("orientation", C.c_uint8),
        ("pad", C.c_uint8 * 7),
    ]


class CDngColour(C.Structure):
    _fields_ = [
        ("temperature", C.c_double),
        ("color_matrix", C.c_double * 9),
        ("forward_matrix", C.c_double * 9),
        ("as_shot_neutral", C.c_double * 3),
        ("baseline_exposure", C.c_double),
        ("illuminant", C.c_uint16),
        ("pad", C.c_uint8 * 6),
    ]


DNG_CODE_VALUES, DNG_LINEAR = 0, 1
DNG_UNCOMPRESSED, DNG_LJ92 = 0, 1

SCALE_FULL = 0

_lib = None


def exported_names():
    """Function names declared in include/prr.h."""
    src = open(HEADER_PATH).read()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(prr_\w+)\s*\(", src, re.M)))


def lib():
    """Load libprr.so; raise if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: the CUDA library must be built "
            "(python -m proresraw_rs_b200.build); there is no CPU fallback"
        )
    L = C.CDLL(LIB_PATH)
    vp, sz, i = C.c_void_p, C.c_size_t, C.c_int
    P = C.POINTER
    sig = {
        "prr_ctx_create": (i, [i, vp, P(vp)]),
        "prr_ctx_destroy": (None, [vp]),
        "prr_ctx_stream": (vp, [vp]),
        "prr_sync": (i, [vp]),
        "prr_status_string": (C.c_char_p, [i]),
        "prr_last_error_string": (C.c_char_p, [vp]),
        "prr_padded_packet_bytes": (sz, [sz]),
        "prr_kernel_launches": (C.c_uint64, []),
        "prr_header_len": (i, [vp, sz, P(sz), P(CError)]),
        "prr_parse_header": (i, [vp, sz, P(CHeader), P(CError)]),
        "prr_frame_info_parse": (i, [vp, sz, P(CFrameInfo), P(CError)]),
        "prr_parse_frame": (i, [vp, sz, P(CFrameInfo), P(C.c_uint8), P(CError)]),
        "prr_decode": (i, [vp, vp, sz, i, vp, sz, P(CDecodeResult), P(CError)]),
        "prr_decode_reduced": (i, [vp, vp, sz, i, i, vp, sz, P(CDecodeResult), P(CError)]),
        "prr_decode_scratch_bytes": (sz, [P(CFrameInfo)]),
        "prr_decode_async": (i, [vp, P(CFrameInfo), vp, i, vp, vp, vp, vp, sz]),
        "prr_decode_reduced_async": (i, [vp, P(CFrameInfo), vp, i, i, vp, vp, vp, vp, sz]),
        "prr_linearize": (i, [vp, P(CHeader), vp, vp, sz]),
        "prr_params_new": (i, [P(CHeader), C.c_uint32, P(CParams)]),
        "prr_params_with_white_balance": (i, [P(CHeader), C.c_uint32, C.c_float, C.c_float, P(CParams)]),
        "prr_output_matrix": (i, [P(CHeader), i, vp]),
        "prr_develop": (i, [vp, P(CHeader), P(CParams), i, vp, i, vp, vp, vp, sz]),
        "prr_develop_set_occupancy": (i, [vp, C.c_uint32]),
        "prr_develop_bucket": (C.c_uint32, [C.c_uint32, C.c_uint32]),
        "prr_develop_set_config": (i, [vp, C.c_uint32, P(CDevelopConfig)]),
        "prr_develop_get_config": (i, [vp, C.c_uint32, P(CDevelopConfig)]),
        "prr_develop_tune": (i, [vp, P(CHeader), P(CParams), i, vp, i, vp, vp, vp, sz, C.c_uint32,
                                 P(CDevelopConfig), P(C.c_float)]),
        "prr_decode_develop_host": (i, [vp, vp, sz, i, P(CParams), i, i, vp, vp, vp, sz, P(CDecodeResult),
                                        P(CError)]),
        "prr_transform_blocks": (i, [vp, i, vp, vp, vp, sz]),
        "prr_decode_components": (i, [vp, vp, vp, vp, sz, i, i, vp]),
        "prr_decode_components_events": (i, [vp, vp, vp, vp, sz, i, i, i, vp, vp, vp]),
        "prr_div_rn_pairs": (i, [vp, vp, vp, vp, sz]),
        "prr_div_rn_check": (i, [vp, C.c_uint32, C.c_uint32, vp]),
        "prr_sqrt_rn_check": (i, [vp, i, i, vp]),
        "prr_decode_noalloc": (i, [i, vp, P(CFrameInfo), vp, i, vp, vp, vp]),
        "prr_batch_submit": (i, [vp, P(CJob), sz]),
        "prr_batch_wait": (i, [vp, C.c_uint32]),
        "prr_batch_set_wait_limit": (i, [vp, C.c_uint32]),
        "prr_batch_drop_chunk_for_test": (i, [vp, C.c_uint32]),
        "prr_batch_last_ms": (i, [vp, P(C.c_float)]),
        "prr_batch_bucket": (i, [vp, P(CJob), sz, P(C.c_uint32)]),
        "prr_batch_tune": (i, [vp, P(CJob), sz, C.c_uint32, P(CBatchConfig), P(C.c_float)]),
        "prr_batch_set_config": (i, [vp, C.c_uint32, P(CBatchConfig)]),
        "prr_batch_get_config": (i, [vp, C.c_uint32, P(CBatchConfig)]),
        "prr_sg_param_count": (sz, []),
        "prr_develop_learned": (i, [vp, P(CHeader), P(CParams), i, vp, P(CSgModel), i, vp, vp, vp, sz,
                                    P(C.c_uint32)]),
        "prr_sg_trainer_create": (i, [vp, C.c_uint32, C.c_uint32, P(vp)]),
        "prr_sg_trainer_destroy": (None, [vp]),
        "prr_sg_trainer_add_frame": (i, [vp, P(CHeader), P(CParams), vp, P(C.c_uint32)]),
        "prr_sg_trainer_noise_range": (i, [vp, P(C.c_float), P(C.c_float)]),
        "prr_sg_trainer_set_params": (i, [vp, vp]),
        "prr_sg_trainer_get_params": (i, [vp, vp]),
        "prr_sg_trainer_device_params": (vp, [vp]),
        "prr_sg_trainer_step": (i, [vp, vp, C.c_float, P(C.c_float)]),
        "prr_sg_pack": (i, [vp, P(CHeader), P(CParams), i, vp, vp, vp]),
        "prr_sg_gradients": (i, [vp, vp, vp, vp, C.c_uint32, C.c_uint32, vp, vp, vp, P(C.c_double)]),
        "prr_mov_open": (i, [C.c_char_p, MOV_ACCEPT_FN, vp, P(vp), C.c_char_p, sz]),
        "prr_mov_close": (None, [vp]),
        "prr_mov_get_info": (i, [vp, P(CMovInfo)]),
        "prr_mov_get_samples": (i, [vp, sz, sz, P(CMovSample)]),
        "prr_mov_warning": (C.c_char_p, [vp, sz]),
        "prr_mov_metadata": (i, [vp, sz, P(C.c_char_p), P(C.c_char_p)]),
        "prr_mov_read_at": (i, [vp, C.c_uint64, vp, sz, C.c_char_p, sz]),
        "prr_clip_create": (i, [i, vp, C.c_uint32, C.c_uint32, P(vp)]),
        "prr_clip_create_fd": (i, [i, i, P(CMovSample), sz, C.c_uint32, C.c_uint32, P(vp)]),
        "prr_clip_destroy": (None, [vp]),
        "prr_clip_start": (i, [vp, C.c_uint64, C.c_uint64, i, i, i]),
        "prr_clip_queue": (i, [vp, C.c_uint64, C.c_uint64, i, i, i]),
        "prr_clip_next": (i, [vp, P(CClipBatch)]),
        "prr_clip_last_error": (C.c_char_p, [vp]),
        "prr_lj92_tile_bound": (C.c_uint64, [C.c_uint32]),
        "prr_lj92_encode": (i, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, vp, C.c_uint64, vp]),
        "prr_lj92_encode_host": (i, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, vp, sz, vp,
                                     P(sz)]),
        "prr_dng_write": (i, [vp, P(CHeader), vp, i, i, P(CDngClip), P(vp)]),
        "prr_dng_write_into": (i, [vp, P(CHeader), vp, i, i, P(CDngClip), vp, sz, P(sz)]),
        "prr_dng_assemble": (i, [P(CHeader), P(CDngClip), i, i, vp, vp, sz, P(vp)]),
        "prr_dng_data": (P(C.c_uint8), [vp, P(sz)]),
        "prr_dng_free": (None, [vp]),
        "prr_dng_colour_of": (i, [P(CHeader), P(CDngColour)]),
        "prr_dng_srational": (i, [C.c_double, P(C.c_int32), P(C.c_int32)]),
        "prr_dng_rational": (i, [C.c_double, P(C.c_uint32), P(C.c_uint32)]),
        "prr_dng_date_time": (i, [C.c_uint64, C.c_char_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L
