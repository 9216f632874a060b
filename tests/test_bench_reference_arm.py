"""The benchmark's reference arm on the host: it must time the CPU
restatement of the reference's path without loading the fusion library (its
configuration comes from plain numbers, its frames from the generator), on
exactly the --warmup / --steps frames the GPU arm times, and print one JSON
line with the reference arm's keys."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, sys
sys.path.insert(0, ROOT)
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1"]
import bench
rc = bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"rc": rc, "fusion_module": any(m.startswith("fusion_b200") for m in sys.modules),
                  "fusion_so": "libfusion_b200" in maps,
                  "so": sorted({l.split()[-1].split("/repo/")[-1] for l in maps.splitlines()
                                if l.endswith(".so") and "/repo/" in l})}))
"""


def test_reference_arm_loads_no_fusion_library():
    env = dict(os.environ, RANK="0", CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", PROBE.replace("ROOT", repr(ROOT))], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    line, probe = json.loads(lines[0]), json.loads(lines[-1])
    assert probe["rc"] == 0
    assert not probe["fusion_module"], "the reference arm imported fusion_b200"
    assert not probe["fusion_so"], "the reference arm mapped libfusion_b200.so"
    assert all(p.startswith(("oracle/", "rgbd_synth/")) for p in probe["so"]), probe["so"]
    assert line["impl"] == "reference"
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["unit"] == "frames/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
