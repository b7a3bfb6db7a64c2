"""The reference arm of bench.py must run the reference alone: its scene set-up (orbit, scene
centre, processing-velocity polynomial) comes from the oracle's FP64 restatement, and the process
never maps a library of this repository.  Checked on the CPU in a fresh interpreter, against the
same scene prepared through the library (both arms must focus the same scene)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

import asarf
from asarf import scene as S

ROOT = Path(__file__).resolve().parent.parent

_CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import bench
sc = bench.make_scene("ers_full", 1001)
sc.prepare(geometry=bench.OracleGeometry())
print(json.dumps({{"vr_poly": list(sc.vr_poly), "center": list(sc.center_point),
                  "first_line_time_us": sc.first_line_time_us, "libs": bench._mapped_native_libs()}}))
"""


def test_reference_arm_scene_set_up_loads_no_library_of_this_repository():
    out = subprocess.run([sys.executable, "-c", _CHILD.format(root=str(ROOT))], capture_output=True, text=True,
                         cwd=ROOT, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    got = json.loads(out.stdout.strip().splitlines()[-1])
    assert got["libs"] == []
    sc = S.WORKLOADS["ers_full"](seed=1001)
    sc.prepare(asarf.load_library())
    x = np.arange(0, sc.range_size, 97)
    assert np.allclose(np.polyval(got["vr_poly"], x), np.polyval(sc.vr_poly, x), rtol=1e-9, atol=0)
    assert np.allclose(got["center"], sc.center_point, rtol=0, atol=1e-3)
    assert got["first_line_time_us"] == sc.first_line_time_us
