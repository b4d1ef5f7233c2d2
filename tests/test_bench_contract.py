"""bench.py's output contract, checked on CPU: the reference arm (the CPU
restatement on the host cores) prints one JSON line with the keys the bench
contract names and never loads the CUDA library, and the GPU arm without a GPU
fails instead of falling back to a CPU path."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# bench.py run in-process, then the libraries the process mapped are listed
_WRAP = ("import runpy, sys\n"
         "sys.argv = ['bench.py'] + sys.argv[1:]\n"
         "rc = 0\n"
         "try:\n"
         "    runpy.run_path('bench.py', run_name='__main__')\n"
         "except SystemExit as e:\n"
         "    rc = e.code or 0\n"
         "maps = open('/proc/self/maps').read()\n"
         "print('MAPPED ' + ('product' if 'libspectral_cuda' in maps else 'none'))\n"
         "sys.exit(rc)\n")


def _run(*args):
    return subprocess.run([sys.executable, "-c", _WRAP, *args], capture_output=True, text=True, cwd=ROOT,
                          timeout=600)


@pytest.mark.parametrize("workload", ["prism", "tracer", "batch", "serve", "split"])
def test_reference_arm_prints_one_contract_line(workload):
    r = _run("--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "1", "--cpu-seconds", "0.5")
    assert r.returncode == 0, r.stderr[-2000:]
    # the reference arm times the CPU restatement only: the product library stays unloaded
    assert "MAPPED none" in r.stdout, r.stdout[-500:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["higher_is_better"] is True and d["vs_baseline"] is None and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    if workload == "prism":  # the reference's serial photon loop, timed beside the threaded one
        assert d["cpu_baseline"]["serial"]["cores"] == 1 and d["cpu_baseline"]["serial"]["value"] > 0
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_gpu_arm_without_a_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = _run("--workload", "prism", "--steps", "1", "--warmup", "1", "--no-cpu-baseline")
    assert r.returncode != 0 and not any(ln.startswith("{") for ln in r.stdout.splitlines())
