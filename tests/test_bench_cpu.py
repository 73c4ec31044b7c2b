"""bench.py's CPU parts without a GPU: the reference arm's JSON line (the
reference build, or the oracle port where it is absent) and the bounded
CPU samples of the workloads."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--workload", "csg4m"], capture_output=True, text=True, timeout=600,
                       cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "samples/s"
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_cpu_samples_keep_the_workload_geometry():
    sys.path.insert(0, str(ROOT))
    import bench
    a = bench.cpu_scene("heldout16m", 2000)
    b = bench.cpu_scene("heldout16m", 2000)
    assert a.n == 2000 and a.k == 1
    np.testing.assert_array_equal(a.pos, b.pos)          # seeded
    assert a.cams.shape[0] >= 64
    assert (a.scale > 0).all() and a.links.max() < a.cams.shape[0]
