"""bench.py --impl reference on the CPU: the reference algorithm (the oracle
port of the Fortran, on all host threads) over the benchmark's own mesh,
built by the oracle's restatement of the reference's mesh set-up, so the
arm loads no library of the product; its JSON line carries the contract's
keys, the timed unit and the host CPU."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

SCRIPT = r'''
import io, json, sys, contextlib
sys.path.insert(0, sys.argv[1])
sys.argv = ["bench.py", "--impl", "reference", "--case", "c1", "--steps", "1", "--warmup", "0"]
import bench
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    rc = bench.main()
maps = [l.split()[-1] for l in open("/proc/self/maps") if ".so" in l]
print(json.dumps({"rc": rc, "line": buf.getvalue().strip().splitlines()[-1],
                  "libs": sorted({m for m in maps if "nim" in m})}))
'''


def test_reference_arm_uses_only_the_oracle():
    out = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["rc"] == 0
    line = json.loads(res["line"])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "cpu_baseline", "e2e", "host_cpu", "per_step_work_ms", "timed_unit"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
    # the oracle's library and nothing of the product's
    assert res["libs"] and all("libnim_oracle" in m for m in res["libs"]), res["libs"]
