"""The server's scheduler (admission by footprint, continuous batching, arrival order, latency
summary) checked on the host with a fake executor: compiles tests/serve_sched_check.cpp against
the library's own scheduler header and runs it. No GPU."""
from __future__ import annotations

import os
import subprocess

from conftest import REPO


def test_scheduler_host_checks(tmp_path):
    exe = str(tmp_path / "serve_sched_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", os.path.join(REPO, "include"),
                    "-I", os.path.join(REPO, "cracklingplusplus_gpu_b200", "csrc"),
                    os.path.join(REPO, "tests", "serve_sched_check.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().endswith("ok")
