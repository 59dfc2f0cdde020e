"""Copy the reference's example inputs (examples/input.cfg, dots.cfg,
pulse.cfg) into tests/golden/ as parity fixtures.

These are the only inputs the reference ships.  With c0*dt = 1.5 um and all
dots inside +-0.1 um, every pair has floor delay 0, so the example exercises
the current-step coupling that the corrector iterations re-evaluate.

Usage (needs the reference checkout): python tests/golden/make_example_fixture.py REF_ROOT
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_example_fixture.py REF_ROOT  (the reference project's root directory)")
    ref = sys.argv[1]
    for name in ["input.cfg", "dots.cfg", "pulse.cfg"]:
        src = os.path.join(ref, "examples", name)
        dst = os.path.join(HERE, "example_" + name)
        shutil.copyfile(src, dst)
        print("wrote", dst)


if __name__ == "__main__":
    main()
