"""The benchmark's reference arm builds and renders its workload on the CPU
without the library (CPU only): the oracle's host generator and threaded
pack make the cloud, and the library's shared object is never loaded."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--points", "300000", "--width", "320",
            "--height", "180", "--steps", "2", "--warmup", "1", "--poses", "4"]
sys.path.insert(0, ".")
import bench
out = bench.run_reference(bench.parse_args(), bench.Dist())
maps = open("/proc/self/maps").read()
print(json.dumps({"line": out,
                  "package_imported": any(m.startswith("satin-computerasteriser_b200")
                                          for m in sys.modules),
                  "library_mapped": "libsatincr" in maps}))
"""


def test_reference_arm_runs_without_the_library():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert not res["package_imported"]
    assert not res["library_mapped"]
    line = res["line"]
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "Gpts/s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port"
