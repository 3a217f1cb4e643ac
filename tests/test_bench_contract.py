"""The reference arm of bench.py on CPU: one JSON line with the contract's
keys, timed by full renders of the CPU restatement of the reference's
renderer on the scaled config-2 scene (no GPU needed); the targets summary
of the GPU line."""
import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def _last_json_line(text):
    lines = [line for line in text.splitlines() if line.startswith("{")]
    assert lines, text[-2000:]
    return json.loads(lines[-1])


def test_reference_arm_prints_the_contract_line():
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
           "--cpu-processes", "1"]
    proc = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    line = _last_json_line(proc.stdout)
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["unit"] == "Mrays/s" and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0.0
    assert "workload" in line["config"]
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] == 1 and cpu["value"] == line["value"]
    assert "48x32 render at 1 spp per process" in cpu["sample"] and "nothing extrapolated" in cpu["sample"]
    assert line["config"]["triangles"] == 5138 and line["config"]["max_bounces"] == 8
    # the timed steps' time is the run's own: no extrapolation
    assert line["ms_per_step"] * line["steps"] < 600e3
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_a_cpu_step_renders_every_bounce_of_the_scaled_scene(tmp_path):
    """One step is a full render per process: the camera rays of a 48x32
    image plus its extension segments, all traced (nothing scaled)."""
    code = (
        f"import sys; sys.path.insert(0, {str(REPO)!r})\n"
        "import bench\n"
        "if __name__ == '__main__':\n"
        "    ref = bench.CpuReference(1)\n"
        "    try:\n"
        "        rays, secs = ref.run_step()\n"
        "    finally:\n"
        "        ref.close()\n"
        "    print(rays, secs)\n"
    )
    # spawned pool workers re-import the main module, so it must be a file
    script = tmp_path / "sample_probe.py"
    script.write_text(code)
    proc = subprocess.run([sys.executable, str(script)], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    rays, secs = proc.stdout.split()[-2:]
    assert int(rays) > 48 * 32 and float(secs) > 0.0


def test_targets_summary_gathers_the_north_star_ratios():
    sys.path.insert(0, str(REPO))
    import bench

    line = {"config1": {"gpu_over_cpu": 900.0, "e2e_over_cpu": 700.0},
            "scaled_c2": {"gpu_mrays_closest_hit": 4000.0}, "cpu_baseline": {"value": 0.02},
            "batched": {"speedup_vs_plain_frame": 8.0, "speedup_vs_plain_resident": 1.1},
            "served": {"rate_req_s": 200.0, "speedup_mrays_vs_plain_frame": 5.0,
                       "speedup_mrays_vs_plain_resident": 1.0, "p50_ms": 30.0, "p99_ms": 150.0, "rejected": 0}}
    t = bench.targets_summary(line)
    assert t["config1_gpu_over_cpu"] == 900.0 and t["config1_required"] == 100.0
    assert t["scaled_c2_gpu_over_cpu"] == 4000.0 / 0.02
    assert t["served_speedup_vs_plain_frame"] == 5.0 and t["systems_required"] == 3.0
