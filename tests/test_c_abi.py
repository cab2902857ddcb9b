"""include/prr.h from C: a C11 program (tests/c_abi/host_calls.c), compiled
with -Wall -Wextra -pedantic -Werror against the header and linked to
lib/libprr.so, makes the host-side calls on a synthetic packet; its answers
must be the Python mirror's (no GPU needed)."""

import os
import shutil
import subprocess

import numpy as np
import pytest

import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib
from proresraw_rs_b200 import dng as D
from proresraw_rs_b200 import synth as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.dirname(_lib.LIB_PATH)


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    out = str(tmp_path_factory.mktemp("c_abi") / "host_calls")
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi", "host_calls.c"), "-o", out, "-L", LIB_DIR, "-lprr",
                    f"-Wl,-rpath,{LIB_DIR}"], check=True)
    return out


def f32(text):
    # %.9g in C round-trips a float32 exactly.
    return [np.float32(float(v)) for v in text.split(",")]


def run(program, packet, tmp_path):
    path = tmp_path / "frame.prr"
    path.write_bytes(packet)
    res = subprocess.run([program, str(path)], check=True, capture_output=True, text=True)
    return dict(line.split("=", 1) for line in res.stdout.splitlines())


@pytest.mark.parametrize("pattern,version", [(S.RGGB, 1), (S.BGGR, 0), (1, 1)])
def test_host_calls_from_c_match_python(program, tmp_path, pattern, version):
    m = S.mosaic(600, 400, pattern, seed=3, sigma=8.0, white=4095)
    spec = S.Spec(600, 400, pattern=pattern, alignment=2, white_level=4095, version=version, valid_tiles=True,
                  wb=(1.7, 1.3), color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
    pkt = S.encode(spec, m, qscale=(15, 45), qscale_seed=7)
    got = run(program, pkt, tmp_path)
    assert got["header_len_rc"] == "0" and int(got["header_len"]) == P.header_len(pkt)
    parsed = P.parse_frame(pkt)
    info = P.frame_info(pkt)
    h = parsed.header
    assert got["parse_frame_rc"] == "0"
    assert (int(got["width"]), int(got["height"])) == (h.width, h.height)
    assert (int(got["coded_width"]), int(got["coded_height"])) == (info.coded_width, info.coded_height)
    assert (int(got["ntiles"]), int(got["tiles_per_row"]), int(got["tile_rows"])) == (
        info.ntiles, info.tiles_per_row, info.tile_rows)
    assert int(got["bayer"]) == int(h.bayer_pattern) and int(got["white"]) == h.white_level
    assert int(got["max_qscale"]) == parsed.max_qscale
    prm = P.DemosaicParams.new(h, P.frame_quantizer(parsed))
    c = prm._c()
    assert got["params_rc"] == "0"
    assert int(got["cfa_phase"]) == c.cfa_phase and int(got["black"]) == c.black
    assert f32(got["one_over_range"]) == [np.float32(c.one_over_range)]
    assert f32(got["noise"]) == [np.float32(v) for v in c.noise]
    assert f32(got["clip"]) == [np.float32(v) for v in c.clip]
    assert f32(got["wb"]) == [np.float32(v) for v in c.wb]
    assert f32(got["matrix"]) == [np.float32(v) for v in P.output_matrix(h).reshape(-1)]
    assert int(got["truncated_rc"]) < 0 and got["truncated_code"] == got["truncated_rc"]
    assert got["status"] == _lib.lib().prr_status_string(int(got["truncated_rc"])).decode()
    assert got["srational"] == "%d/%d" % D.srational(-0.3125)
    assert got["rational"] == "%d/%d" % D.rational(2.2)
    assert got["date"] == D.quicktime_date_time(3000000000)
    assert int(got["padded_100"]) == _lib.lib().prr_padded_packet_bytes(100)
    assert int(got["lj92_bound_256"]) == _lib.lib().prr_lj92_tile_bound(256)
