"""bench.py's reference arm on the CPU: one JSON line with the contract's
keys for one rank, and for two ranks under torch.distributed.run exactly one
line (rank 0 works, the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")
ARGS = ["--impl", "reference", "--workload", "single", "--steps", "1", "--warmup", "3"]


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check(line):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"]
    e = line["e2e"]
    assert e["value"] == line["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_one_rank():
    r = subprocess.run([sys.executable, BENCH] + ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0])


def test_reference_arm_two_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), BENCH, "--gpus", "2"] + ARGS
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0])
    assert lines[0]["n_gpus"] == 2


def test_reference_arm_loads_no_product_code():
    """The reference arm's processes load the reference's own library
    (oracle/_ref) or the C restatement, never libmbt.so."""
    code = (
        "import os, sys, tempfile; sys.path.insert(0, %r)\n"
        "import bench\n"
        "conf = bench.conf_path('single', tempfile.mkdtemp())\n"
        "nb, npb = bench._ring_probe(conf)\n"
        "t = bench._cpu_worker((bench.cpu_kind(), conf, 0, nb, 1))\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('libmbt.so' in maps, 'libmbtref.so' in maps or 'liboracle.so' in maps, nb, len(t))\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split()[-4:] == ["False", "True", "1", "1"], r.stdout
