"""CPU tests of bench.py's host-side legs: the reference arm runs the oracle only (the
CUDA library is never loaded in its process) and its line describes what ran."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpu_legs_do_not_load_the_library():
    code = (
        "import sys, bench\n"
        "legs = bench.cpu_oracle_legs(1, n3_solve=False)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED' if 'libfame_b200' in maps or 'fame_b200' in sys.modules else 'CLEAN')\n"
        "print(legs['action']['iters'] > 0)\n"
    )
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["CLEAN", "True"], out.stdout


def test_reference_arm_line():
    """--impl reference at N=1: value = mean step x 40 Lanczos steps (labelled
    extrapolated), ms_per_step = the measured step, plus a measured N=3 solve."""
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--N", "1", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["extrapolated"] is True
    cb = line["cpu_baseline"]
    assert abs(line["value"] - cb["action_seconds"] * 40) < 0.01 + 1e-3 * line["value"]
    assert abs(line["ms_per_step"] - 1e3 * cb["action_seconds"]) < 1.0
    assert cb["n3_full_solve_s"] > 0 and cb["n3_lanczos_steps"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
