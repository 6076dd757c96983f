"""bench.py's reference arm (the reference's own CPU path, host only) prints
one JSON line with the contract's keys, on the default workload's config."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(*args, timeout=600):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True,
                       text=True, timeout=timeout, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_harness.so")),
                    reason="the reference library is built where its sources are (oracle/_ref)")
def test_reference_arm_line():
    line = run("--impl", "reference", "--steps", "4", "--warmup", "0", "--ref-sweep", "none")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["config"]["workload"] == "mixed_streams_48"
    assert line["metric"] == "Mpix-frames/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["steps"] == 4 and line["warmup"] == 0
    per = line["cpu_baseline"]["per_size"]
    assert sorted(per) == ["1280x720", "1920x1080", "3840x2160", "640x480"]
    for v in per.values():
        assert v["mpix_frames_s"] > 0 and v["preseed_ms"] > 0 and v["frames_timed"] >= 8


@pytest.mark.parametrize("workload", ["served_poisson", "served_saturated"])
def test_served_reference_arm_is_unavailable(workload):
    line = run("--impl", "reference", "--workload", workload)
    assert line["impl"] == "reference" and "unavailable" in line


def test_clock_sampler_samples_before_the_timed_region(tmp_path, monkeypatch):
    """The clock sampler's nvidia-smi is started and has written its first
    sample before the timed region begins; its summary gives the median SM
    clock, the max clock and the active throttle reasons (a fake nvidia-smi
    on PATH, no GPU)."""
    fake = tmp_path / "nvidia-smi"
    fake.write_text(
        "#!/bin/sh\n"
        "sleep 0.3\n"
        "while true; do\n"
        "  echo '0, 1965, 1965, 700.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active'\n"
        "  sleep 0.05\n"
        "done\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ.get('PATH', '')}")
    sys.path.insert(0, ROOT)
    try:
        import bench
    finally:
        sys.path.remove(ROOT)
    with bench.ClockSampler(0) as c:
        assert c.proc is not None and os.path.getsize(c.path) > 0   # first sample already in
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] >= 1
