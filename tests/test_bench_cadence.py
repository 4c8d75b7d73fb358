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


@pytest.mark.parametrize("W,K,up,warm,total", [(5, 20, 100, 1, 21), (100, 500, 100, 100, 600), (250, 20, 100, 200, 220),
                                              (20, 21, 20, 20, 41), (3, 2, 100, 1, 3)])
def test_reference_cadence(W, K, up, warm, total):
    import bench
    assert bench.reference_cadence(W, K, up) == (warm, total)


# Stands in for the reference's mem_cuda: the same steady-timer rule (cuda/mem_cuda.cu:1859,
# 1912-1920: the timer starts inside a diagnostic step it == 1, it % UPDATE == 0 or it == STEPS,
# once it >= BENCH_WARMUP_STEPS) and the same end-of-run lines (:2024-2036).
FAKE_MEM_CUDA = r'''#!/usr/bin/env python3
import os, sys
steps, update = int(sys.argv[4]), int(sys.argv[6])
warm = int(os.environ.get("BENCH_WARMUP_STEPS", str(update)))
start = 0 if warm <= 0 else None
for it in range(1, steps + 1):
    if it == 1 or it % update == 0 or it == steps:
        print(" ITERATION %6d T=0" % it)
        if start is None and it >= warm:
            start = it
print(" Frames per second (FPS)            = %12.7f" % 500.0)
if start is not None and steps - start > 0:
    print(" Steady frames per second (FPS)     = %12.7f  (%d steps after warmup)" % (530.25, steps - start))
    print(" Steady FPS: %12.7f" % 530.25)
print("[OUTPUT] Normal completion; no output files written.")
'''


def _fake(tmp_path):
    exe = tmp_path / "mem_cuda"
    exe.write_text(FAKE_MEM_CUDA)
    exe.chmod(0o755)
    return str(exe)


def test_reference_arm_window_with_short_warmup(tmp_path):
    """--steps 20 --warmup 5 at UPDATE=100: the reference's steady window covers exactly 20 steps."""
    import bench
    warm, total = bench.reference_cadence(5, 20, 100)
    v, steady, _ = bench.run_reference_binary(_fake(tmp_path), [4096, "1E+05", 4, total, 0.1, 100, 0], warm,
                                              str(tmp_path))
    assert steady == 20 and v == pytest.approx(530.25)


def test_reference_arm_reports_why_it_has_no_window(tmp_path):
    """Passing the warm-up straight through (the old rule) leaves no steady window; the error
    says which line is missing instead of 'failed rc=0'."""
    import bench
    with pytest.raises(RuntimeError, match="no 'Steady frames per second' line"):
        bench.run_reference_binary(_fake(tmp_path), [4096, "1E+05", 4, 25, 0.1, 100, 0], 5, str(tmp_path))


def test_parse_reference_stdout():
    import bench
    out = (" Frames per second (FPS)            =  512.1234567\n"
           " Steady frames per second (FPS)     =  530.7654321  (500 steps after warmup)\n"
           " Steady FPS:  530.7654321\n")
    assert bench.parse_reference_stdout(out) == (pytest.approx(530.7654321), 500)
    assert bench.parse_reference_stdout(" FPS: 1.0\n") is None


def test_window_plan():
    import bench
    assert bench.window_plan(5, 20, 100, 0.6) == [5 + 20 * i for i in range(84)]
    assert bench.window_plan(100, 500, 100, 0.6) == [100, 600, 1100, 1600]
    assert len(bench.window_plan(5, 20, 100, 1e-9)) == 200


def test_reference_arm_initial_field(tmp_path):
    """The reference arm's restart.bin: the workload's seeded k^4 field at step 0 with the FP64
    oracle's NEXTDT-init dt, in the v2 layout the reference's loader reads (a small N here)."""
    import struct
    import numpy as np
    import bench
    from oracle import oracle as O
    bench.select_workload("dns4096", 32)
    try:
        path = str(tmp_path / "restart.bin")
        note = bench.reference_initial_field(32, path)
        assert "k^4" in note
        b = open(path, "rb").read()
        h = struct.unpack("<16s4I10i9f4x4Q", b[:144])
        assert h[5] == 32 and h[13] == 0 and h[19] > 0  # N, it, dt
        om = np.frombuffer(b, dtype=np.complex64, count=32 * 16, offset=144 + 3 * 48 * 48 * 4).reshape(32, 16)
        assert np.array_equal(om, O.k4_spectrum(32, 4.0, 0))
    finally:
        bench.select_workload("dns4096", None)


def test_network_trace_summary():
    """The persistent network launch's trace summary: per-layer spans and per-step medians of a
    synthetic trace (2 layers of 2 tile rows x 1 strip, 2 CTAs, every step 100 ns apart)."""
    import numpy as np
    import bench
    tiles = 4
    tr = np.zeros((tiles, 10), dtype=np.uint64)
    for i in range(tiles):
        tr[i] = 1000 + 500 * i + 100 * np.arange(10)
    out = bench.network_trace_summary(tr, 3, 2, 1, 2)
    assert out["tiles"] == 4 and out["ctas"] == 2
    assert out["span_us"] == round((1500 + 900) / 1e3, 2)
    assert [l["layer"] for l in out["layers"]] == [1, 2]
    assert all(v == 0.1 for v in out["layers"][0]["median_us"].values())
    assert out["layers"][1]["first_taken_us"] == 1.0 and out["layers"][1]["last_released_us"] == 2.4
    assert out["tile_interval_per_cta_us"] == 1.0
