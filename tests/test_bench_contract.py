"""The reference arm of bench.py on CPU: one JSON line with the contract's
keys, timed by the CPU restatement of the reference's brute-force
intersector (no GPU needed)."""
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
           "--cpu-processes", "1", "--reference-seconds", "1"]
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
    assert "64x64-pixel tile" in cpu["sample"] and "scaled to all of them" in cpu["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_cpu_sample_scales_a_triangle_block_to_the_scene(tmp_path):
    """The sampled block's time is scaled by (all triangles / block): two
    block sizes of the same tile give scaled times of one order."""
    code = (
        f"import sys; sys.path.insert(0, {str(REPO)!r})\n"
        "import bench\n"
        "if __name__ == '__main__':\n"
        "    ref = bench.CpuReference(1)\n"
        "    try:\n"
        "        r1, s1 = ref.run_step(triangles=512)\n"
        "        r2, s2 = ref.run_step(triangles=2048)\n"
        "    finally:\n"
        "        ref.close()\n"
        "    print(r1, s1, r2, s2)\n"
    )
    # spawned pool workers re-import the main module, so it must be a file
    script = tmp_path / "sample_probe.py"
    script.write_text(code)
    proc = subprocess.run([sys.executable, str(script)], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    r1, s1, r2, s2 = proc.stdout.split()[-4:]
    assert int(r1) == int(r2) == 64 * 64
    s1, s2 = float(s1), float(s2)
    assert s1 > 0.0 and s2 > 0.0
    assert 0.25 < s1 / s2 < 4.0
