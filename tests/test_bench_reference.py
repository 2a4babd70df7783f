"""The benchmark's reference arm (`bench.py --impl reference`) on the host
cores: one JSON line with the contract's keys, no GPU needed."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# Run inside the arm's process after it printed its line: the product library
# must not be mapped (the arm times the reference's code, not this engine's).
_PROBE = """
import runpy, sys
sys.argv = ["bench.py"] + sys.argv[1:]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit:
    pass
maps = open("/proc/self/maps").read()
print("PRODUCT_MAPPED" if "librayengine_b200" in maps else "PRODUCT_NOT_MAPPED")
print("REF_MAPPED" if "libre_ref" in maps else "REF_NOT_MAPPED")
"""


@pytest.mark.parametrize("config", ["soup", "terrain_sdf"])
def test_reference_arm_prints_one_contract_line(config):
    out = subprocess.run([sys.executable, "-c", _PROBE, "--impl", "reference",
                          "--config", config, "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "Mrays/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["warmup"] >= 3
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "PRODUCT_NOT_MAPPED" in out.stdout
    if config == "soup" and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libre_ref.so")):
        # meshes: the reference's own compiled CPU query is what is timed,
        # over the configured SAH tree, with the as-shipped one-leaf tree
        # beside it
        assert d["cpu_baseline"]["kind"] == "reference" and "REF_MAPPED" in out.stdout
        assert "SAH kd-tree of the configured parameters" in d["cpu_baseline"]["sample"]
        assert 0 < d["as_shipped"]["value"] < d["value"]
