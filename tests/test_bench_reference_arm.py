"""The bench's reference arm (``bench.py --impl reference``) on the CPU: it times the oracle, prints one
JSON line whose ``config`` equals the one the GPU arm prints for the same workload, and never maps the
product library (the package loads libablate_fv.so on the first ABI call only, and the arm makes none).
Run on a 16^3 Taylor-Green box so that it takes seconds.
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

DRIVER = """
import sys
sys.path.insert(0, {root!r})
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3", "--n", "16"]
import bench
rc = bench.main()
maps = open("/proc/self/maps").read()
print("MAPPED", int("libablate_fv" in maps), "RC", rc)
"""


def test_reference_arm_shares_the_config_and_maps_no_product_library():
    out = subprocess.run([sys.executable, "-c", DRIVER.format(root=str(ROOT))], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["value"] > 0
    tail = [l for l in out.stdout.splitlines() if l.startswith("MAPPED")][0].split()
    assert tail[1] == "0", "the reference arm mapped libablate_fv.so"

    sys.path.insert(0, str(ROOT))
    import bench
    from ablate_b200 import workloads
    assert line["config"] == json.loads(json.dumps(bench.workload_config(workloads.tgv3d(16), 1)))
