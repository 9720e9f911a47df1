"""Generate the text fixtures (*.npz) of this directory with the
reference's own psstest.

oracle/_ref/psstest is the reference psstest (src/psstest.cpp) built from the
reference sources by oracle/Makefile. For each text it loads the file as
psstest does (src/tools/input.hpp:255-297), builds the string pointer array
(src/psstest.cpp:479-518), sorts with pS5 (bingmann/parallel_sample_sortBTCUI)
and writes the sorted strings with -o, one per line (psstest.cpp:696-703).
A fixture stores the text, the mode and that output.

Run from the repository root after building:
python tests/golden/text/make_text_golden.py
The fixtures travel without the reference tree.
"""
from __future__ import annotations

import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent.parent
PSSTEST = ROOT / "oracle" / "_ref" / "psstest"


def texts():
    rng = np.random.default_rng(21)
    lines = []
    for _ in range(3000):
        ln = bytes(rng.choice(np.frombuffer(b"ab\r", np.uint8), int(rng.integers(0, 13)),
                              p=[0.48, 0.48, 0.04]))
        if rng.random() < 0.02:
            ln += b"\0" + ln[:3]  # a NUL inside a line ends a string too
        lines.append(ln)
    yield "text_lines_mixed", b"\n".join(lines), False  # no trailing newline
    pre = [bytes(rng.integers(97, 123, 40, dtype=np.uint8)) for _ in range(5)]
    lines = [pre[int(rng.integers(0, 5))][: int(rng.integers(0, 41))]
             + bytes(rng.integers(97, 100, int(rng.integers(0, 6)), dtype=np.uint8))
             for _ in range(2500)]
    yield "text_lines_prefixes", b"\n".join(lines) + b"\n", False
    dna = bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), 1600))
    dna = dna[:500] + b"\n" + dna[500:1200] + dna[500:700] + b"\n" + dna[1200:]
    yield "text_suffix_dna", dna, True
    yield "text_lines_tiny", b"hello", False
    yield "text_lines_only_newlines", b"\n\n\n", False


def main():
    with tempfile.TemporaryDirectory() as d:
        for name, text, suffix in texts():
            src = Path(d) / f"{name}.txt"
            out = Path(d) / f"{name}.out"
            src.write_bytes(text)
            cmd = [str(PSSTEST), "-A", "bingmann/parallel_sample_sortBTCUI", "-o", str(out)]
            if suffix:
                cmd.append("--suffix")
            cmd.append(str(src))
            subprocess.run(cmd, check=True, capture_output=True, timeout=300)
            np.savez_compressed(HERE / f"{name}.npz",
                                text=np.frombuffer(text, np.uint8),
                                suffix=np.array(suffix),
                                output=np.frombuffer(out.read_bytes(), np.uint8))
            print(name, len(text), "bytes ->", out.stat().st_size, "bytes of sorted output")


if __name__ == "__main__":
    main()
