"""bench.py's profiling cases (--save-state / --load-state) and small-problem
comparison (--small), run as the profiles' commands run them: a state saved
mid-run reloads into the same solver state, and fin_advance and a batch of
one give the same vortex state bit for bit."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _bench(*args, timeout=600):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                       text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


def test_saved_state_reloads_and_steps(tmp_path):
    path = str(tmp_path / "r64.npz")
    (saved,) = _bench("--forms", "hybrid", "--n", "64", "--window-t", "0.05", "--save-state", path)
    assert saved["steps"] > 0 and abs(saved["t"] - 0.05) < 1e-12
    z = np.load(path)
    assert int(z["n"]) == 64 and z["q"].shape == (70, 70, 5) and np.isfinite(z["q"]).all()
    (run,) = _bench("--forms", "hybrid", "--n", "64", "--load-state", path, "--steps", "2", "--warmup", "3")
    assert run["steps"] == 2 and run["t_start"] == pytest.approx(0.05, abs=1e-12)
    assert run["stage_kernel_ms"] > 0 and run["indicator_kernel_ms"] > 0
    # a state of another size is refused with a message, not run
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--forms", "hybrid", "--n", "128",
                        "--load-state", path], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "pass --n 64" in (r.stdout + r.stderr)


def test_small_problems_advance_equals_batch_of_one():
    rows = _bench("--small")
    assert [r["grid"] for r in rows] == ["64x64", "200x200", "512x512"]
    for r in rows:
        assert r["bitwise_equal"] and r["steps"] == r["batch_steps"] > 0
    assert rows[1]["steps"] == 1464   # the 200^2 vortex to t = 10, as the reference's own run
