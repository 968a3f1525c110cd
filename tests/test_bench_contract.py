"""The benchmark's reference arm (CPU, no GPU needed) keeps its JSON contract."""

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_line(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setattr(bench, "CPU_SAMPLE_SIZES", (2, 3))  # a quick sample for the test
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "1",
                                      "--warmup", "3", "--count", "16"])
    assert bench.main() == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["unit"] == "mol/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1 and "sample" in line["cpu_baseline"]
    assert line["e2e"] == {"value": line["value"], "unit": "mol/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["metric"] == json.loads((ROOT / "BASELINE.json").read_text())["metric"]
