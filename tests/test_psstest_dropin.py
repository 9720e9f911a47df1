"""GPU test of the drop-in boundary inside the reference's own harness.

oracle/_ref/psstest is the reference's psstest (src/psstest.cpp) built from
its sources with the B200 contestants linked in (oracle/Makefile). psstest
checks every run itself: the permutation hash and strcmp order
(src/tools/checker.hpp:131-153), verify_lcp for the LCP contestant and
verify_lcp_cache for the LCP + cache contestant (src/psstest.cpp:659-686),
and reports status=ok only when they pass. The distinguishing prefix and LCP
sum it prints are functions of the sorted sequence, so they must equal pS5's
on the same input.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
PSSTEST = ROOT / "oracle" / "_ref" / "psstest"

GPU_CONTESTANTS = ["gpu/sample_sort", "gpu/sample_sort_lcp", "gpu/sample_sort_lcp_cache",
                   "gpu/sample_sort_out"]


def run_psstest(path, algo, suffix=False):
    cmd = [str(PSSTEST), "-A", algo]
    if suffix:
        cmd.append("--suffix")
    cmd.append(str(path))
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    results = []
    for line in out.stdout.splitlines():
        if line.startswith("RESULT"):
            results.append(dict(kv.split("=", 1) for kv in line.split("\t")[1:] if "=" in kv))
    assert results, out.stdout[-2000:]
    return results[-1]


def write_lines(path, chars, nchars):
    data = chars[:nchars].copy()
    data[data == 0] = 10  # NUL -> newline: psstest's plain-file format
    path.write_bytes(data.tobytes())


@pytest.fixture(scope="module")
def inputs(pkg, tmp_path_factory):
    d = tmp_path_factory.mktemp("psstest")
    c, o, n = pkg.workloads.digits(seed=1)
    digits = d / "digits_10mib.txt"
    write_lines(digits, c, n)
    c, o, n = pkg.workloads.prefixes(n=400000, seed=7)
    prefixes = d / "prefixes_400k.txt"
    write_lines(prefixes, c, n)
    text = pkg.workloads.dna_text(length=4 << 20, seed=3)
    dna = d / "dna_4mib.txt"
    dna.write_bytes(text[: (4 << 20)].tobytes() + b"\n")
    return {"digits": digits, "prefixes": prefixes, "dna": dna}


@pytest.mark.parametrize("name,suffix", [("digits", False), ("prefixes", False), ("dna", True)])
def test_psstest_checks_gpu_contestants(inputs, name, suffix):
    assert PSSTEST.exists(), "oracle/_ref/psstest is built by __graft_entry__.build()"
    ref = run_psstest(inputs[name], "bingmann/parallel_sample_sortBTCUI", suffix)
    assert ref["status"] == "ok"
    ref_out = run_psstest(inputs[name], "bingmann/parallel_sample_sortBTCUI_out", suffix)
    assert ref_out["status"] == "ok"
    assert (ref_out["dprefix"], ref_out["lcpsum"]) == (ref["dprefix"], ref["lcpsum"])
    for algo in GPU_CONTESTANTS:
        r = run_psstest(inputs[name], algo, suffix)
        assert r["status"] == "ok", (algo, r)
        assert r["algo"] == algo
        assert r["string_count"] == ref["string_count"]
        assert r["dprefix"] == ref["dprefix"], (algo, r["dprefix"], ref["dprefix"])
        assert r["lcpsum"] == ref["lcpsum"], (algo, r["lcpsum"], ref["lcpsum"])
