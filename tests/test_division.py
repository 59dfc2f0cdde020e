"""The reciprocal-and-correction division of the dot-step kernels equals
IEEE division (checked on the host: every operation is correctly rounded on
both, so the bits agree)."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_markstein_division_is_exact(tmp_path):
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    exe = tmp_path / "markstein_check"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-o", str(exe),
                    os.path.join(HERE, "native", "markstein_check.c"), "-lm"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout
    assert "mismatches 0" in out.stdout
