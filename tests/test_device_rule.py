"""The one-device rule of the runtime, on the host: objects stay on the device that was current
when they were created, and a call made with another device current is rejected with
PG_ERR_INVALID_ARGUMENT before any device work (pg::check_same_device, which require_same_device
applies to geometry and scenes). Compiled from the runtime's own source with g++; no GPU needed."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(os.path.join(CUDA, "include")),
                    reason="needs g++ and the CUDA headers")
def test_calls_from_another_device_are_rejected(tmp_path):
    exe = tmp_path / "device_check"
    src = os.path.join(ROOT, "photon-v2_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", src, "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "native", "device_check.cpp"),
                    os.path.join(src, "pg_runtime.cpp"), "-L", os.path.join(CUDA, "lib64"), "-lcudart",
                    "-pthread", "-o", str(exe)], check=True)
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(CUDA, "lib64") + os.pathsep + os.environ.get("LD_LIBRARY_PATH", ""))
    out = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
