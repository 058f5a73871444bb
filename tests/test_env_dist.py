"""Environment importance-sampling tables of the physical estimator, on
the CPU: the library's builder (cupbr_b200/csrc/env_dist.hpp) and the
oracle's restatement give bit-identical CDFs, densities and row cosines,
and the density integrates to one over the sphere, for a sky with a sun, a
black map, single-row and single-column maps and a random map."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from cupbr_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("env") / "env_dist_harness")
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-ffp-contract=off", "-D_USE_MATH_DEFINES",
           "-I", os.path.join(ROOT, "cupbr_b200", "csrc"), os.path.join(HERE, "env_dist_harness.cpp"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


CASES = {
    "sky": lambda: scenes.sky_env(128, 64, sun_radiance=500.0),
    "black": lambda: np.zeros((16, 32, 3), np.float32),
    "one_row": lambda: np.random.default_rng(1).random((1, 40, 3)).astype(np.float32),
    "one_column": lambda: np.random.default_rng(2).random((24, 1, 3)).astype(np.float32),
    "random": lambda: (np.random.default_rng(3).random((33, 65, 3)) ** 4).astype(np.float32),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tables_match_the_oracle_and_integrate_to_one(harness, tmp_path, name):
    env = np.ascontiguousarray(CASES[name](), np.float32)
    h, w, _ = env.shape
    path = tmp_path / "env.bin"
    with open(path, "wb") as f:
        np.array([w, h], np.uint32).tofile(f)
        env.tofile(f)
    p = subprocess.run([harness, str(path)], capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    total = float(p.stdout.split()[1])
    if name == "black":
        assert total == 0.0
    else:
        assert abs(total - 1.0) < 1e-5, total
