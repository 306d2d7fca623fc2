"""Host-side checks of bench.py (no GPU): the synthetic workloads match
their stated shapes, and every DRAM-traffic figure the bench line reports
comes from a committed ncu summary that holds the same numbers."""
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_serve_stream_matches_its_description():
    """16 jobs, batch 256..8192 (log-uniform), world 16^3 or 32^3, 32x32 or
    64x64 images, episodes of 200..2000 steps; the same stream every run."""
    jobs = bench.serve_jobs()
    assert jobs == bench.serve_jobs()
    assert len(jobs) == 16
    for j in jobs:
        assert 256 <= j["batch"] <= 8192
        assert j["world"] in (16, 32)
        assert j["res"] in (32, 64)
        assert 200 <= j["episode"] <= 2000
    assert list(bench.SERVE_LOADS) == sorted(bench.SERVE_LOADS)
    assert 0.85 in bench.SERVE_LOADS


def test_workloads():
    assert (bench.WORKLOAD["batch_size"], bench.WORKLOAD["world"], bench.WORKLOAD["res"]) == (32768, 16, 32)
    assert (bench.RENDER_WORKLOAD["batch_size"], bench.RENDER_WORKLOAD["world"],
            bench.RENDER_WORKLOAD["res"]) == (4096, 32, 64)
    assert sum(b for b, _, _ in bench.RAGGED_GROUPS) == 24576


def test_traffic_figures_come_from_committed_profiles():
    for name, (traffic, source) in bench.TRAFFIC.items():
        path = re.search(r"profiles/\S+\.md", source).group(0)
        text = open(os.path.join(ROOT, path)).read()
        # the summary holds the read and write megabytes whose sum is reported
        pairs = [(float(r), float(w)) for r, w in re.findall(r"(\d+\.\d) (?:MB )?/ (\d+\.\d) MB", text)]
        assert any(abs((r + w) * 1e6 - traffic) < 0.05e6 for r, w in pairs), (name, path, traffic)


def test_help_runs_without_a_gpu():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    assert "--workload" in out.stdout
