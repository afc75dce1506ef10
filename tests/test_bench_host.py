"""bench.py's host-side plumbing on CPU: the rank launcher and the batch
sharding of ``--gpus N`` (two gloo ranks), the WORLD_SIZE check under an
external launcher, and the reference arm, which must run the reference's
kernels on the benchmark state without mapping this repository's library."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def _env(**extra):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env.update(extra)
    return env


def test_gpus_2_launches_two_ranks_with_disjoint_blocks():
    r = subprocess.run([sys.executable, BENCH, "--gpus", "2", "--plan-only", "--batch-systems", "24"],
                       capture_output=True, text=True, timeout=300, env=_env(), cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    out = json.loads(lines[0])
    assert out["world"] == 2
    blocks = sorted((b[1], b[2]) for b in out["plan"])
    assert sorted(b[0] for b in out["plan"]) == [0, 1]
    assert blocks[0][0] == 0 and blocks[0][1] == blocks[1][0] and blocks[1][1] == 24
    assert all(b[1] > b[0] for b in blocks)


def test_world_size_must_match_gpus():
    r = subprocess.run([sys.executable, BENCH, "--gpus", "2", "--plan-only"], capture_output=True, text=True,
                       timeout=120, env=_env(WORLD_SIZE="1", RANK="0", LOCAL_RANK="0"), cwd=ROOT)
    assert r.returncode != 0
    assert "WORLD_SIZE=1" in r.stderr


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_reference_arm_runs_without_the_product_library():
    code = ("import runpy, sys\n"
            f"sys.argv = [{BENCH!r}, '--impl', 'reference', '--steps', '1', '--warmup', '1']\n"
            "try:\n"
            f"    runpy.run_path({BENCH!r}, run_name='__main__')\n"
            "except SystemExit:\n"
            "    pass\n"
            "print('MAPPED' if 'libcudaring' in open('/proc/self/maps').read() else 'NOT_MAPPED')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=_env(),
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "NOT_MAPPED"
    line = json.loads([ln for ln in lines if ln.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["state"] == "bench_state/smooth_lj_1024.npz"
    assert line["config"]["workload"].startswith("1024 deformable rings")


def test_clock_sampler_keeps_only_samples_of_the_timed_region(tmp_path, monkeypatch):
    # a stand-in nvidia-smi: one idle-clock line at start-up, then load clocks
    # every interval, the power cap active on the third of them
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/usr/bin/env python3\n"
                    "import sys, time\n"
                    "print('0, 345, 1965, 80.0, 0x0, Not Active, Not Active, Not Active, Not Active', flush=True)\n"
                    "k = 0\n"
                    "while True:\n"
                    "    time.sleep(0.05)\n"
                    "    k += 1\n"
                    "    cap = 'Active' if k == 3 else 'Not Active'\n"
                    "    print(f'0, 1965, 1965, 900.0, 0x4, Not Active, Not Active, Not Active, {cap}', flush=True)\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    monkeypatch.syspath_prepend(ROOT)
    import importlib
    import time
    bench = importlib.import_module("bench")
    with bench.ClockSampler(0) as cs:
        time.sleep(0.6)
    out = cs.summary()
    assert out["samples"] >= 3
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0  # the idle start-up sample is left out
    assert out["reasons"] == ["sw_power_cap"]
