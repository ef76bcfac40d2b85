"""Transcribe the reference's safe-math golden bit patterns into a JSON fixture.

Reads tests/test_safe_math_golden.inc of the reference (Roundabout; the
table generated by its tools/gen_safe_math_golden.F90 from contraction-off
builds) and writes tests/golden/safe_math_golden.json with the CBRT, ATAN,
EXP, LOG and ERFC rows, each [argument_bits, result_bits], and the POW and POWBIG
rows, each [x_bits, y_bits, result_bits], as 16-hex-digit IEEE binary64 words.  These pin the oracle's port of rdb_sm_cbrt / rdb_sm_atan /
rdb_sm_exp / rdb_sm_log / rdb_sm_pow / rdb_sm_erfc bit for bit.

Usage (in a container where the reference tree is mounted):
    python tests/golden/make_safe_math_golden.py /path/to/roundabout
"""
import json
import re
import sys
from pathlib import Path


def parse(inc_text, name):
    m = re.search(r"character\(len=16\), parameter :: G_%s\((\d), NG_%s\) = reshape\(\["
                  r"character\(len=16\) :: &(.*?)\], \[\d, NG_%s\]\)" % (name, name, name),
                  inc_text, re.S)
    if not m:
        raise SystemExit("table %s not found" % name)
    width = int(m.group(1))
    words = re.findall(r'"([0-9A-F]{16})"', m.group(2))
    assert len(words) % width == 0
    return [words[i:i + width] for i in range(0, len(words), width)]


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    text = (ref / "tests" / "test_safe_math_golden.inc").read_text()
    out = {"source": "tests/test_safe_math_golden.inc (reference)",
           "cbrt": parse(text, "CBRT"), "atan": parse(text, "ATAN"), "exp": parse(text, "EXP"),
           "log": parse(text, "LOG"), "pow": parse(text, "POW"), "powbig": parse(text, "POWBIG"),
           "erfc": parse(text, "ERFC")}
    dst = Path(__file__).with_name("safe_math_golden.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", dst, {k: len(v) for k, v in out.items() if isinstance(v, list)})


if __name__ == "__main__":
    main()
