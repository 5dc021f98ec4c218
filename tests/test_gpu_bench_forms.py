"""bench.py's timed forms end to end on the small 128^3 workload (4096-ray batches): each run
exits 0 and prints one JSON line with the keys of the bench contract.  The default plain FP32
line at full size is the round-end run itself; these cover the other forms' code paths (the
proposal's label and guided batches, the mid-run window of --start-batch)."""
import json
import pathlib
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parent.parent
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks"}


@pytest.mark.parametrize("extra", [
    ["--precision", "bf16"],
    ["--precision", "bf16", "--form", "proposal"],
    ["--precision", "bf16", "--form", "proposal", "--start-batch", "130"],
], ids=["mixed", "proposal", "proposal-mid-run"])
def test_bench_form_prints_its_line(cuda, extra):
    cmd = [sys.executable, "bench.py", "--workload", "small128", "--steps", "3", "--warmup", "3",
           "--no-cpu-baseline", *extra]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert KEYS <= set(line), KEYS - set(line)
    assert line["value"] > 0 and line["e2e"]["value"] > 0 and line["gpu_launches"] > 0
    assert line["config"]["precision"] == "bf16"
    if "proposal" in extra:
        assert line["proposal"]["error_flags"] == 0 and line["proposal"]["rounds"] >= 3
        assert line["warmup"] >= (130 if "--start-batch" in extra else 110)
