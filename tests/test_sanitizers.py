"""The host code under AddressSanitizer and UndefinedBehaviorSanitizer (gcc):
the plan compiler of libpsgcuda.so (processseg_b200/csrc/psg_plan.cpp, pure
host C++) and the CPU oracle, driven by tests/sanitize_harness.cpp over every
op kind, both dtypes, invalid parameters and ragged rows. The device code is
checked by its own bounds (the kernels' bounded waits and status word) and
the parity tests; compute-sanitizer is not used on this pool."""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_code_is_clean_under_asan_and_ubsan():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "harness")
        cmd = ["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
               "-fno-omit-frame-pointer", "-I", os.path.join(ROOT, "include"),
               os.path.join(ROOT, "tests", "sanitize_harness.cpp"),
               os.path.join(ROOT, "processseg_b200", "csrc", "psg_plan.cpp"),
               os.path.join(ROOT, "oracle", "psg_oracle.cpp"), "-o", exe, "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-4000:]
        env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
                   UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
        r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
        assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]
        assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-4000:]
