"""bench.py's reference arm on the CPU (no GPU needed): the oracle timed on a
sample of the batch, printing the contract's JSON line with impl
"reference", its cpu_baseline and a zero-copy e2e."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run(
        [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scenes", "16", "--steps",
         "1", "--warmup", "1", "--preroll", "1", "--sample-stride", "4"],
        capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "body-substeps/s"
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["scenes"] == 16
