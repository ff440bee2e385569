"""Host logic of bench.py that needs no GPU: the partition of the wavelength
sweep over the timed steps (every wavelength weighted equally whatever
--steps is), the reference arm's operator-application table and its refusal
to extrapolate outside it, and the profile figures the JSON line quotes."""
import json
import math
import os
import subprocess
import sys
from collections import Counter

import pytest

import bench
from tests.conftest import ROOT


@pytest.mark.parametrize("steps", [1, 3, 7, 20, 51, 52, 60])
def test_sweep_plan_weights_every_wavelength_equally(steps):
    plan, reps = bench.sweep_plan(51, steps)
    assert len(plan) == steps
    assert reps == math.ceil(steps / 51)
    counts = Counter(i for step in plan for i in step)
    assert set(counts) == set(range(51))
    assert set(counts.values()) == {reps}
    sizes = [len(step) for step in plan]
    assert max(sizes) - min(sizes) <= 1  # the solves spread evenly over the steps


def test_warmup_plan_one_solve_per_step():
    warm = bench.warmup_plan(51, 3)
    assert len(warm) == 3 and all(len(w) == 1 and 0 <= w[0] < 51 for w in warm)


def test_sweep_is_the_configuration_grid():
    assert len(bench.SWEEP_NM) == 51
    assert bench.SWEEP_NM[0] == 400.0 and bench.SWEEP_NM[-1] == 900.0


def test_reference_counts_cover_the_sweep_only():
    counts = bench.reference_counts(30000, 1e-8)
    assert counts is not None and set(counts) == set(bench.SWEEP_NM)
    assert all(c > 0 for c in counts.values())
    assert bench.reference_counts(6000, 1e-8) is None
    assert bench.reference_counts(30000, 1e-6) is None


def test_reference_arm_refuses_other_configurations():
    """Outside the counted configuration the reference arm prints its
    unavailable line and exits 0 rather than guessing a count."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--size", "10,10,10", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and "unavailable" in line
    assert "N=1000" in line["unavailable"]


def test_profile_traffic_figures_are_readable():
    assert bench._traffic_from_profiles("otf_pairs_f32_sym") > 0
    assert bench._traffic_from_profiles("gemv_dense_blocks", "cuboid6k") > 1e9
    assert bench._traffic_from_profiles("no_such_kernel") is None
