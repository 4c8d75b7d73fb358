"""bench.py host logic on the CPU: the step segments of its diagnostic cadence (which it prepares
as graphs before timing) are the segments advance() runs, and the ensemble workload's reference
arm reports that the reference has no ensemble."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


class _Recorder:
    """Stands in for a Solver: records the segment lengths advance() asks for."""

    def __init__(self, it=0):
        self.it, self.calls, self.diag = it, [], []

    def scalars(self):
        return {"it": self.it}

    def step(self, n, history=False):
        self.calls.append(n)
        self.it += n
        return None

    def next_dt(self):
        self.diag.append(self.it)

    def om2phys(self):
        pass

    def display_sigma(self, comp):
        return 0.0


@pytest.mark.parametrize("it0,it1,up", [(0, 500, 100), (100, 600, 100), (3, 53, 100), (0, 41, 20), (20, 41, 20)])
def test_segments_are_what_advance_runs(it0, it1, up):
    import bench
    r = _Recorder(it0)
    bench.advance(r, it1, up, it1, {"kernels": 0})
    assert r.calls == bench.segments(it0, it1, up)
    assert sum(r.calls) == it1 - it0
    # a diagnostic (NEXTDT) after step 1, every multiple of UPDATE and the last step
    assert all(d == 1 or d % up == 0 or d == it1 for d in r.diag)


def test_ensemble_reference_arm_is_unavailable():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--workload", "ensemble", "--impl",
                          "reference"], capture_output=True, text=True, timeout=120, cwd=REPO)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
