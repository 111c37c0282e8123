"""bench.py's plumbing on the CPU: `--gpus N` without an outer torchrun starts N ranks itself, and the reference arm
(the oracle timed on the host cores) loads none of the product's native code and prints the same workload config as
the GPU arm."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out: str) -> dict:
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert lines, out
    return json.loads(lines[-1])


def _env():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    return env


def test_gpus_n_starts_n_ranks_without_an_outer_launcher():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"], cwd=ROOT,
                       env=_env(), capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stdout + r.stderr
    line = _last_json(r.stdout)
    assert line["n_gpus"] == 2 and line["ranks_joined"] == 2
    assert line["config"]["parallelism"] == "replicas x2"


def test_reference_arm_loads_only_the_oracle_and_prints_the_same_config():
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED', 'libhush_b200' in maps, 'liboracle_hush' in maps)\n"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=_env(), capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "LOADED False True" in r.stdout, r.stdout
    line = _last_json(r.stdout)
    assert line["impl"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0
    sys.path.insert(0, ROOT)
    import bench

    assert line["config"] == bench._config("fp32", 1)
