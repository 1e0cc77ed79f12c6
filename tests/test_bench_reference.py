"""The bench's reference arm on the CPU: it times the oracle (the
reference algorithm's CPU restatement) on inputs made without libvt.so --
the torch restatement of the seeded generators and the oracle's octree
builder -- and its line carries the same `config` as the product arm's."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, sys, types
sys.path.insert(0, %r)
import torch, bench
args = types.SimpleNamespace(steps=1, warmup=3, ref_budget=0.3, ref_total=2.0, config="c1")
line = bench.run_reference(args, bench.CONFIGS["c1"], 0, 1, torch)
maps = open("/proc/self/maps").read()
print(json.dumps({"line": line, "libvt": "libvt.so" in maps, "oracle": "liboracle.so" in maps,
                  "conf": bench.workload_config(bench.CONFIGS["c1"], "c1", 1)}))
"""


def test_reference_arm_runs_without_libvt():
    r = subprocess.run([sys.executable, "-c", PROBE % ROOT], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["libvt"], "the reference arm loaded libvt.so"
    assert out["oracle"]
    line = out["line"]
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "rays/s"
    assert line["config"] == out["conf"]
    assert line["cpu_baseline"]["kind"] == "port" and "vs CPU port" in line["note"]
