"""CPU check of the FP64 NTT butterfly schedule (signed twiddles, one
normalisation per round of up to four stages): exact against 128-bit modular
arithmetic, with every magnitude precondition of the proof in csrc/ntt.cuh
asserted, on random and adversarial inputs. The C program performs the
kernel's own IEEE double operations, so a pass here means the device path
computes the same residues."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "fp64_butterfly_bounds.c")


def test_fp64_butterfly_schedule(tmp_path):
    exe = tmp_path / "fp64_butterfly_bounds"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), SRC, "-lm"], check=True)
    r = subprocess.run([str(exe), "60000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "violations=0 mismatches=0" in r.stdout
