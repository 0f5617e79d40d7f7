"""Golden outputs of the reference's own test programs, linked with the
reference's own sources (oracle/_ref/ref_<program>, built by
oracle/build_ref.sh) and run on a B200: tests/golden/ref_programs/<program>.txt.

tests/test_ref_programs_gpu.py runs the same programs linked against this
library and requires every result line (errors, mismatch counts, PASS lines;
clock lines are skipped) to be identical to these. Run on a GPU machine:
    python tests/golden/make_ref_program_golden.py
"""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(ROOT, "tests", "golden", "ref_programs")
PROGRAMS = ["test_stage_acc", "test_keyreuse", "test_chain", "test_rot_resident", "test_boot"]


def main():
    os.makedirs(OUT, exist_ok=True)
    for p in PROGRAMS:
        exe = os.path.join(REF, "ref_" + p)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=1800, cwd=REF)
        if r.returncode != 0:
            raise SystemExit(f"{p}: exit {r.returncode}\n{r.stdout[-2000:]}{r.stderr[-2000:]}")
        with open(os.path.join(OUT, p + ".txt"), "w") as f:
            f.write(r.stdout)
        print(p, "ok")


if __name__ == "__main__":
    main()
