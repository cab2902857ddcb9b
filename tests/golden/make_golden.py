"""Copies the reference crate's golden IDCT data into tests/golden/.

The proresraw_rs crate pins its Apple-compatible IDCT with two files
(src/idct.rs:562-594): tests/data/idct_vectors.bin, 512 records of
(i16[64] coefficients, i16[64] quantizers, u16[64] expected code values),
little-endian, and tests/data/idct_hash.txt, the FNV-1a hash of the outputs
of 2^20 blocks from testgen::Gen(0x4a54). They are data, copied verbatim so
the tests can run where the reference tree is absent.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
(REFERENCE_ROOT: the proresraw_rs checkout, the directory holding tests/data/)
"""
import hashlib
import pathlib
import shutil
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py REFERENCE_ROOT")
root = pathlib.Path(sys.argv[1])
here = pathlib.Path(__file__).resolve().parent
for name in ["idct_vectors.bin", "idct_hash.txt"]:
    src = root / "tests" / "data" / name
    shutil.copyfile(src, here / name)
    print(name, hashlib.sha256((here / name).read_bytes()).hexdigest())
