"""The backend adapter (nemosim_b200/adapter/b200_backend.cpp): the two
symbols libnemo resolves from its dynamically loaded CUDA backend that take
the reference's C++ classes, cuda_simulation and cuda_set_configuration
(src/nemo/cuda/create_simulation.hpp:16-20, src/nemo/cuda/devices.cpp:225-246).

The adapter is compiled here against stand-ins of the reference headers
that declare the signatures it implements (tests/adapter/include; the
reference headers need Boost), linked with the native library and driven by
tests/adapter/driver.cpp through the nemo::SimulationBackend interface only,
as libnemo drives a backend: the reference's ring, current-stimulus and STDP
known-answer tests on a GPU, and the configuration and creation errors
without one."""
import os
import shutil
import subprocess

import pytest

import nemosim_b200 as nb
from nemosim_b200 import build as nbuild

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def compile_driver(out_dir) -> str:
    nb.lib()  # the native library is built
    exe = os.path.join(str(out_dir), "adapter_driver")
    libdir = os.path.dirname(nbuild.LIB)
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-Wno-unused-parameter",
           "-I", os.path.join(HERE, "adapter", "include"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "nemosim_b200", "adapter", "b200_backend.cpp"),
           os.path.join(HERE, "adapter", "standins.cpp"), os.path.join(HERE, "adapter", "driver.cpp"),
           "-L", libdir, "-lnemo_b200", "-Wl,-rpath," + libdir, "-o", exe]
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    assert res.returncode == 0, res.stdout + res.stderr
    return exe


def run(exe, mode):
    res = subprocess.run([exe, mode], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0 and res.stdout.strip() == "ok", res.stdout + res.stderr


def test_adapter_compiles_and_fails_cleanly_without_a_device(tmp_path):
    from tests.conftest import HAS_GPU
    exe = compile_driver(tmp_path)
    if HAS_GPU:
        pytest.skip("a device is present: the GPU test drives the adapter")
    run(exe, "nodevice")


@pytest.mark.gpu
def test_adapter_runs_the_reference_known_answer_tests(tmp_path):
    run(compile_driver(tmp_path), "gpu")
