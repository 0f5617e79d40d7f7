"""The reference's own test programs, compiled unchanged against this library.

tests/cpp/build_ref_programs.sh compiles five of the reference's OpenFHE-free
test programs (tests/test_rot_resident.cpp, test_keyreuse.cpp, test_chain.cpp,
test_stage_acc.cpp, test_boot.cpp) from their own sources against include/
and libgpufhe_b200.so, with no source change: a caller of the reference
relinks and runs. Each program checks itself and prints [PASS] / [FAIL]; the
test requires exit status 0 and the [PASS] line, and that the program loaded
this library. Where the same program linked against the reference's own
sources was run on a B200 (tests/golden/ref_programs/*.txt, made by
tests/golden/make_ref_program_golden.py), every line that carries a result
(errors, mismatch counts, PASS lines, not clocks) must be identical.
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "ref_programs")
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_programs")
LIB = os.path.join(ROOT, "gpu-resident-library_b200", "gpufhe_b200", "libgpufhe_b200.so")

PROGRAMS = ["test_stage_acc", "test_keyreuse", "test_chain", "test_rot_resident", "test_boot"]

# lines that report a clock or a speed: they differ run to run
TIMING = re.compile(r"(\d\s*s\b|\bms\b|\bsec|x\)|speedup|[0-9]x\b|time|min |med |min/med|GB/s)", re.I)


def result_lines(text):
    return [ln.rstrip() for ln in text.splitlines() if ln.strip() and not TIMING.search(ln)]


@pytest.mark.parametrize("prog", PROGRAMS)
def test_reference_program_passes_on_this_library(prog):
    exe = os.path.join(BIN, prog)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is not built (sh tests/cpp/build_ref_programs.sh REFERENCE_ROOT)")
    ldd = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert os.path.realpath(LIB) in {os.path.realpath(p) for p in re.findall(r"=>\s*(\S+)", ldd)}, ldd
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900, cwd=BIN)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "[PASS]" in r.stdout
    gold = os.path.join(GOLDEN, prog + ".txt")
    if os.path.exists(gold):
        want = result_lines(open(gold).read())
        got = result_lines(r.stdout)
        assert got == want, "\n".join(f"want {w!r}\n got {g!r}" for w, g in zip(want, got) if w != g)
