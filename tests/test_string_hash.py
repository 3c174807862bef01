"""The oracle's qdb_string_hash_bytes (qdb/modules/qumirdb_runtime.cpp:270-300)
for strings of every length: up to 16 bytes against an independent Python
restatement of the engine's short-string formula, above 16 bytes against
XXH3-64 from the xxHash header that Apache Arrow vendors (the engine's own
dependency), with the engine's secret — every length branch of XXH3
(17-128, 129-240, one and several 576-byte blocks) and their edges."""
import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent


def _pin():
    try:
        import pyarrow
    except ImportError:
        pytest.skip("pyarrow (the vendored xxHash header) is not installed")
    inc = Path(pyarrow.__file__).parent / "include"
    if not (inc / "arrow" / "vendored" / "xxhash" / "xxhash.h").exists():
        pytest.skip("pyarrow ships no vendored xxHash header")
    out = Path(tempfile.mkdtemp()) / "xxh3_pin.so"
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", f"-I{inc}", str(ROOT / "oracle" / "xxh3_pin.c"), "-o",
                    str(out)], check=True, capture_output=True)
    lib = C.CDLL(str(out))
    lib.pin_xxh3_with_secret.restype = C.c_uint64
    lib.pin_xxh3_with_secret.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]
    return lib


def _short(b: bytes) -> int:
    m0, m1 = 11400714785074694791, 14029467366897019727
    M = (1 << 64) - 1

    def mix(mul, v):
        return int.from_bytes(((mul * v) & M).to_bytes(8, "little"), "big")

    n = len(b)
    if n == 0:
        return 1
    if n <= 3:
        return mix(m0, (n << 24) ^ (b[0] << 16) ^ (b[n // 2] << 8) ^ b[n - 1])
    if n <= 8:
        x, y = int.from_bytes(b[n - 4:], "little"), int.from_bytes(b[:4], "little")
    else:
        x, y = int.from_bytes(b[n - 8:], "little"), int.from_bytes(b[:8], "little")
    return n ^ mix(m0, x) ^ mix(m1, y)


EDGES = [17, 18, 31, 32, 33, 63, 64, 65, 95, 96, 97, 127, 128, 129, 130, 143, 144, 239, 240, 241, 255, 256,
         511, 575, 576, 577, 640, 1151, 1152, 1153, 1728, 4096, 10_000]


def test_short_strings_match_the_engine_formula():
    rng = np.random.default_rng(1)
    for n in range(0, 17):
        for _ in range(20):
            b = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
            assert O.string_hash(b) == _short(b), (n, b)


def test_long_strings_match_vendored_xxh3():
    pin = _pin()
    secret = O.string_secret()
    assert len(secret) == 136
    sbuf = C.create_string_buffer(secret, len(secret))
    rng = np.random.default_rng(2)
    lengths = EDGES + [int(x) for x in rng.integers(17, 3000, 300)]
    for n in lengths:
        for _ in range(3):
            b = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
            buf = C.create_string_buffer(b, n)
            want = pin.pin_xxh3_with_secret(buf, n, sbuf, 136)
            assert O.string_hash(b) == want, n
    # text-like strings too (a shared prefix, ASCII bytes)
    for n in (20, 100, 200, 700):
        b = (b"https://example.org/" * 50)[:n]
        buf = C.create_string_buffer(b, n)
        assert O.string_hash(b) == pin.pin_xxh3_with_secret(buf, n, sbuf, 136)
