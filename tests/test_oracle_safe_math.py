"""The oracle's port of rdb_sm_cbrt / rdb_sm_atan / rdb_sm_exp / rdb_sm_log / rdb_sm_pow against the reference's
golden bit patterns (tests/test_safe_math_golden.inc, transcribed into
tests/golden/safe_math_golden.json)."""
import json
import struct
from pathlib import Path

import pytest

GOLD = json.loads((Path(__file__).parent / "golden" / "safe_math_golden.json").read_text())


def h2d(s):
    return struct.unpack(">d", bytes.fromhex(s))[0]


def d2h(x):
    return struct.pack(">d", x).hex().upper()


@pytest.mark.parametrize("fn", ["cbrt", "atan", "exp", "log", "erfc"])
def test_golden_bits(oracle, fn):
    f = {"cbrt": oracle.sm_cbrt, "atan": oracle.sm_atan, "exp": oracle.sm_exp, "log": oracle.sm_log,
         "erfc": oracle.sm_erfc}[fn]
    bad = []
    for arg, res in GOLD[fn]:
        got = d2h(f(h2d(arg)))
        if got != res:
            bad.append((arg, res, got))
    assert not bad, f"{len(bad)} of {len(GOLD[fn])} {fn} rows differ: {bad[:4]}"


@pytest.mark.parametrize("table", ["pow", "powbig"])
def test_golden_bits_pow(oracle, table):
    bad = []
    for x, y, res in GOLD[table]:
        got = d2h(oracle.sm_pow(h2d(x), h2d(y)))
        if got != res:
            bad.append((x, y, res, got))
    assert not bad, f"{len(bad)} of {len(GOLD[table])} {table} rows differ: {bad[:4]}"
