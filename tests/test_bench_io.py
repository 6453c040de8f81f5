"""bench.py --config io on the host: the .dat reader's throughput line (and
the reference reader's, femModel::ReadFromFEMTextFile compiled from the
reference sources) keeps the bench JSON contract.  Small mesh; no GPU
needed (the writers are timed only with a device)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*extra):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--config", "io", "--n", "8", "--steps", "2",
                        "--warmup", "1", *extra], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_io_line():
    d = _run("--no-cpu")
    assert d["unit"] == "MB/s" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["higher_is_better"] is True and d["vs_baseline"] is None
    assert "reader of the 8^3 Kuhn-tet cavity" in d["config"]["workload"]
    assert d["read_s"]["min"] > 0


def test_io_reference_line():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/fm_refdrv not built")
    d = _run("--impl", "reference")
    assert d["impl"] == "reference" and d["unit"] == "MB/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 1
    assert d["e2e"]["value"] == d["value"]
