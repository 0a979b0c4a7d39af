"""The benchmark's reference arm (`bench.py --impl reference`) on the CPU: the JSON line it
prints follows the benchmark contract (metric, unit, a cpu_baseline describing the run, an
e2e object with no host-device copies), it times the oracle at the workload's own sizes,
and it loads nothing of the engine (no `aquarius_b200` module, no `libccsd_b200.so`)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import runpy, sys, json
sys.argv = ["bench.py", "--impl", "reference", "--workload", "{workload}", "--steps", "1", "--warmup", "3"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    code = e.code or 0
else:
    code = 0
maps = open("/proc/self/maps").read()
print(json.dumps({{"exit": code, "engine_module": "aquarius_b200" in sys.modules,
                   "engine_so": "libccsd_b200" in maps}}))
"""


def _run(workload):
    out = subprocess.run([sys.executable, "-c", PROBE.format(workload=workload)], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    return json.loads(lines[0]), json.loads(lines[-1])


def test_reference_arm_line_and_isolation():
    line, probe = _run("small")
    assert probe == {"exit": 0, "engine_module": False, "engine_so": False}
    assert line["impl"] == "reference"
    assert line["metric"] == "CCSD iterations/s" and line["unit"] == "iter/s" and line["higher_is_better"]
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] >= 3
    assert line["config"]["o"] == 8 and line["config"]["v"] == 48 and line["config"]["nirrep"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "o=8 v=48" in cb["sample"]   # timed at the workload's own sizes
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # the estimate is the sum over statements of slab time / slab fraction
    assert abs(sum(line["per_statement_s"].values()) - line["est_s_per_iteration"]) <= 1e-9 * line["est_s_per_iteration"]


def test_reference_arm_symmetry_blocked_workload_is_unavailable():
    line, probe = _run("cfg4")
    assert probe["exit"] == 0 and not probe["engine_so"]
    assert line["impl"] == "reference" and "unavailable" in line
