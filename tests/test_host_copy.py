"""CPU check of the host staging helpers (non-temporal copies and the
float64 / int64 conversions of minhashcuda_b200/csrc/host_copy.cc) against
memcpy and scalar casts: compiles tests/host_copy_check.cc with the helpers
and runs it.  Needs g++ and the CUDA headers (the helpers' header includes
cuda_runtime.h)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


@pytest.mark.skipif(shutil.which("g++") is None or
                    not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")),
                    reason="needs g++ and the CUDA headers")
def test_host_copy_helpers_match_scalar_code(tmp_path):
    exe = tmp_path / "host_copy_check"
    subprocess.check_call([
        "g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "minhashcuda_b200", "csrc"),
        "-I", CUDA_INCLUDE, os.path.join(ROOT, "tests", "host_copy_check.cc"),
        os.path.join(ROOT, "minhashcuda_b200", "csrc", "host_copy.cc"), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
