"""The host C of libmbt (mbt_host.c, mbt_beam.c, mbt_output.c,
mbt_ws_output.c: configuration reader, Green's functions, generated beams,
slicing, both writers) under AddressSanitizer and UndefinedBehaviorSanitizer:
tests/host_sanitize_main.c drives them on the test configurations; any bad
access or undefined operation aborts the run."""
import os
import shutil
import subprocess

import pytest

from tests.util import small_conf, slice_conf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mbtrack_b200", "csrc")
SOURCES = ["mbt_host.c", "mbt_beam.c", "mbt_output.c", "mbt_ws_output.c"]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc absent")
def test_host_code_under_sanitizers(tmp_path):
    exe = str(tmp_path / "host_sanitize")
    cmd = (["gcc", "-std=gnu11", "-O1", "-g", "-fno-omit-frame-pointer", "-ffp-contract=off",
            "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-I" + os.path.join(ROOT, "include"),
            os.path.join(ROOT, "tests", "host_sanitize_main.c")]
           + [os.path.join(CSRC, s) for s in SOURCES] + ["-o", exe, "-lm"])
    subprocess.check_call(cmd)
    work = tmp_path / "work"
    work.mkdir()
    weak = [small_conf(tmp_path, n) for n in ("single_bunch.conf", "uniform_fill.conf", "uneven_fill.conf",
                                              "feedback_hc.conf", "beam_ion.conf")]
    strong = [slice_conf(tmp_path, "train"), slice_conf(tmp_path, "gaps")]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe, str(work)] + weak + ["--"] + strong, capture_output=True, text=True, timeout=600,
                       env=env, cwd=ROOT)   # fill files named relative to the repository
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]
    assert "host calls ok" in r.stdout
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr
