"""The C ABI from plain C: tests/c_consumer.c (C99, no C++ or Python) is
compiled with gcc against include/sph3.h and linked to libsph3.so.  On CPU it
must build, load and report that there is no GPU; on a B200 it runs the first
step and two KDK steps of a 4,096-particle sphere and checks the density,
the status word and the mass sum."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    from sph_3_b200 import build as b
    lib = b.build()
    exe = str(tmp_path / "c_consumer")
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c_consumer.c"), "-o", exe, "-L", os.path.dirname(lib), "-lsph3",
           "-Wl,-rpath," + os.path.dirname(lib), "-lm"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def _gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def test_c_consumer_without_gpu(tmp_path):
    if _gpu():
        pytest.skip("a GPU is present")
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "no device", out.stdout + out.stderr


@pytest.mark.gpu
def test_c_consumer_runs_steps(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0 and out.stdout.startswith("ok "), out.stdout + out.stderr
