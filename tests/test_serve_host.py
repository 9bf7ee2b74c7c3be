"""The serving loop's admission policy (fastandfourier_b200/csrc/faf_sched.h)
on the CPU: tests/native/sched_check.cpp is compiled with g++ and run (arena,
FIFO admission, merging, memory budget, streamed-request order, a random
submit/complete fuzz)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_scheduler_policy(tmp_path):
    exe = os.path.join(tmp_path, "sched_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
                    "-I" + os.path.join(ROOT, "fastandfourier_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "sched_check.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "OK"


def test_server_rejects_without_gpu_or_bad_config():
    """faf_server_create fails cleanly (NULL + message) where it cannot run."""
    import fastandfourier_b200 as F
    from fastandfourier_b200 import _lib as C
    if C.lib().faf_cuda_available():
        pytest.skip("a GPU is present; covered by the GPU tests")
    with pytest.raises(F.FafError):
        F.Server(hbm_budget=1 << 20)
