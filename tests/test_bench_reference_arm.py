"""bench.py's reference arm, on the host: its JSON line carries the keys the
bench contract asks for, with the same config as the library's arm, and
its process never maps libbml_b200.so (the arm times the reference
library's own CPU path, with inputs from the oracle's copy of the seeded
generator).  One timed step and no warm-up, so it runs in well under a
minute on a few host cores."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.skipif(not O.available(), reason="oracle/_ref is not built")

RUN = (
    "import runpy, sys\n"
    "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
    "try:\n"
    "    runpy.run_path('bench.py', run_name='__main__')\n"
    "except SystemExit as e:\n"
    "    assert not e.code, e.code\n"
    "maps = open('/proc/self/maps').read()\n"
    "print('MAPPED_LIBRARY_UNDER_TEST', int('libbml_b200' in maps))\n"
)


def test_reference_arm_line_and_mapped_libraries():
    r = subprocess.run([sys.executable, "-c", RUN], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.splitlines()
    assert "MAPPED_LIBRARY_UNDER_TEST 0" in out
    line = json.loads([s for s in out if s.startswith("{")][-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 1 and line["warmup"] == 0
    assert line["value"] > 0 and line["higher_is_better"] is False
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    import bench
    assert line["config"] == bench.bench_config(1)
