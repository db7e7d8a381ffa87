"""The benchmark's reference arm runs the reference's CPU implementation
without this project's GPU library: run on a small frame in a fresh process,
it prints its JSON line and the process never maps libdpb200.so."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys, types
sys.path.insert(0, {root!r})
import bench
bench.N_SIDE = 4  # 192 atoms
bench.run_reference(types.SimpleNamespace(steps=2, warmup=1), 0, 1)
maps = open("/proc/self/maps").read()
print(json.dumps({{"libdpb200": "libdpb200" in maps,
                  "package": any(m.startswith("deepmd_kit_lr_pt_b200") for m in sys.modules)}}))
"""


def test_reference_arm_is_independent_of_the_product():
    out = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["steps"] == 2 and line["unit"] == "us/step/atom"
    assert line["config"]["nloc"] == 192 and line["value"] > 0
    assert abs(line["ms_per_step"] * 1e3 / 192 - line["value"]) < 1e-9 * line["value"]
    assert not probe["libdpb200"] and not probe["package"]
