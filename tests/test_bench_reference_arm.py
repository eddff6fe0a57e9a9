"""bench.py --impl reference: the reference's own CPU implementation of the path
(the programs built from the reference sources under oracle/_ref, or the oracle
port when they are absent) timed on the host, printed as one JSON line with the
same metric and unit as the GPU arm plus the keys the reference arm adds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "active cell-updates/s" and d["unit"] == "cell-updates/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "modelb_2048_fp32_conserved"


def test_reference_arm_dendrite_program():
    """The dendrite workloads time the reference's own CPU_version program when it is built."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "dendrite_512_fp64", "--steps", "4", "--warmup", "0"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert d["impl"] == "reference" and d["value"] > 0 and d["config"]["workload"] == "dendrite_512_fp64"
    built = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "dendrite_cpu"))
    assert d["cpu_baseline"]["kind"] == ("reference" if built else "port")
