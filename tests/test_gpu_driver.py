"""quest-gpu on the reference's example inputs (examples/input.cfg,
dots.cfg, pulse.cfg; committed as tests/golden/example_*.cfg): output.dat in
the reference's format, equal to the library's own trajectory to the 12
printed digits and to the oracle within the FP64 tolerance."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from quest_b200 import capi, inputs as I
from tests.conftest import GOLDEN, ROOT, rel_err

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "quest_b200", "quest-gpu")


def setup_case(tmp_path, num_particles=None, total_time=None):
    for name in ("dots", "pulse"):
        shutil.copy(os.path.join(GOLDEN, f"example_{name}.cfg"), tmp_path / f"{name}.cfg")
    c, n, _, _ = I.read_input_cfg(os.path.join(GOLDEN, "example_input.cfg"))
    if num_particles is not None:
        n = num_particles
    if total_time is not None:
        c.num_timesteps = int(np.ceil(total_time / c.dt))
    I.write_input_cfg(str(tmp_path / "input.cfg"), c, n)
    return c, n


@pytest.mark.parametrize("num_particles,total_time", [(None, None), (1024, 1.0)])
def test_driver_on_the_reference_examples(tmp_path, golden_weights, oracle_weights, num_particles, total_time):
    c, n = setup_case(tmp_path, num_particles, total_time)
    out = subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert out.stdout.splitlines() == ["Initializing...", "Solving...", "Writing output..."]
    got = I.read_output_dat(str(tmp_path / "output.dat"))
    assert got.shape == (c.num_timesteps, n, 2)
    dots = I.read_dots_cfg(str(tmp_path / "dots.cfg"), n)
    pulse = I.read_pulse_cfg(str(tmp_path / "pulse.cfg"))
    with capi.Simulation(dots, pulse, c, weights=golden_weights) as sim:
        ref = sim.run(c.num_timesteps)
    # 13 significant digits printed
    assert rel_err(ref[..., 0], got[..., 0]) < 1e-12 and rel_err(ref[..., 1], got[..., 1]) < 1e-12
    steps = min(c.num_timesteps, 400)
    hist, bad = O.run_fast(dots, pulse, c, oracle_weights, steps)
    assert bad is None
    oref = O.rho_trajectory(hist)
    assert rel_err(oref[..., 0], got[:steps, :, 0]) < 1e-10
    assert rel_err(oref[..., 1], got[:steps, :, 1]) < 1e-10
    # the text layout: one line per step, two "(re,im)" fields per dot
    first = open(tmp_path / "output.dat").readline()
    assert first.count("(") == 2 * n and first.endswith(" \n")


def test_driver_nonfinite_run_writes_no_output(tmp_path):
    c, n = setup_case(tmp_path, 2, 0.05)
    # a dot with T1 = 0 (a zero-initialised dot of a short dots file)
    lines = open(tmp_path / "dots.cfg").read().split("\n")
    open(tmp_path / "dots.cfg", "w").write(lines[0] + "\n")
    out = subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert out.returncode == 1
    assert "std::domain_error" in out.stderr
    assert not (tmp_path / "output.dat").exists()
