"""The reference arm of bench.py (`--impl reference`) on the CPU: it times the
oracle (the C restatement of the reference's CG) on the host cores and prints
one JSON line with the contract's keys, including the one-thread figure and an
e2e entry that moves no bytes across PCIe.  A 16^3 grid keeps it to a second."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "16",
                          "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] >= 3
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["value_1thread"] > 0 and "whole solves" in cb["sample"]
    assert cb["nproc"] >= 1 and cb["logical_cpus"] >= cb["nproc"] and "cpu_model" in cb
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["iterations"] > 0


def test_gpus_n_launches_n_ranks():
    """`bench.py --gpus 2` without a launcher starts two ranks itself (torch.distributed.run on
    127.0.0.1); the ranks join one gloo group and rank 0 prints one line with n_gpus = 2."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "12",
                          "--gpus", "2", "--steps", "1", "--warmup", "3", "--ref-1thread-solves", "0"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2


def test_gpus_mismatch_with_launcher_fails():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "12",
                          "--gpus", "2", "--steps", "1"], capture_output=True, text=True, timeout=120, cwd=ROOT,
                         env=env)
    assert out.returncode == 2 and "WORLD_SIZE=1" in out.stderr
