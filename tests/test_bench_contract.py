"""bench.py's reference arm on CPU: one JSON line with the contract's keys, the
CPU port timed on a bounded sample, exit code 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-views", "2"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["config"]["workload"] == "dd3_proj_back_512x512x256_984v_888x64"
    # measured, not extrapolated: one sampled step, and no CUDA library loaded
    assert d["ms_per_step"] < 600_000
    assert "extrapolated, not run" in d["cpu_baseline"]["sample"]


def test_reference_arm_loads_no_cuda_library():
    """The reference arm draws its scan and phantom without the package: no
    libctlab_b200.so in the process's maps, and the same config dict as our arm."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
            "'--cpu-views', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); print('LOADED' if 'libctlab_b200' in maps else 'CLEAN')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    sys.path.insert(0, ROOT)
    import types
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    ours = bench.config_dict(types.SimpleNamespace(views=0, sat="zprefix"))
    assert d["config"] == ours
