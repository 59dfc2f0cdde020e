"""The reference-compatible command-line driver (quest_b200/quest-gpu): the
checks that need no GPU (command line, configuration errors).  The runs
themselves are in test_gpu_driver.py."""
import os
import subprocess

import pytest

from tests.conftest import ROOT

EXE = os.path.join(ROOT, "quest_b200", "quest-gpu")


def run(args, cwd):
    return subprocess.run([EXE] + args, cwd=cwd, capture_output=True, text=True, timeout=60)


def test_help_lists_the_reference_options(tmp_path):
    out = run(["--help"], tmp_path)
    assert out.returncode == 0
    for key in ("--config", "files.qd_path", "files.pulse_path", "constants.c0", "constants.hbar",
                "constants.mu0", "constants.laser_frequency", "parameters.num_particles",
                "parameters.total_time", "parameters.timestep", "parameters.interpolation_order"):
        assert key in out.stdout, key


def test_version(tmp_path):
    out = run(["-v"], tmp_path)
    assert out.returncode == 0 and "QuEST" in out.stdout


def test_missing_config_is_reported_like_the_reference(tmp_path):
    out = run([], tmp_path)  # default input.cfg, absent
    assert out.returncode == 0 and "ERROR: input.cfg not found" in out.stderr
    assert not (tmp_path / "output.dat").exists()


def test_missing_required_key(tmp_path):
    (tmp_path / "input.cfg").write_text("[parameters]\n  num_particles = 2\n  total_time = 1\n"
                                        "  timestep = 0.01\n  interpolation_order = 3\n")
    out = run([], tmp_path)
    assert out.returncode == 1
    assert "the option 'constants.c0' is required but missing" in out.stderr


@pytest.mark.parametrize("args,msg", [(["--bogus"], "unrecognised option"),
                                      (["--precision", "fp16"], "--precision"),
                                      (["--coefficients"], "missing")])
def test_bad_command_lines(tmp_path, args, msg):
    out = run(args, tmp_path)
    assert out.returncode == 1 and msg in out.stderr
