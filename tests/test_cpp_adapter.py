"""include/csd_cpp.hpp, the header-only C++ adapter with the reference's
host signatures (checkCollisionFreeCuda, cuda_collision_checker.h:93-94;
computeForwardKinematicsCuda, cuda_forward_kinematics.h:53-55;
CudaEdgeInflator, cuda_polytope_builder.h:16-44; ...), compiled with g++
against stand-ins of the reference's types (tests/cpp/adapter_demo.cpp) and
linked to the library. Without a GPU the program checks the error mapping;
with one (-m gpu) it checks verdicts, FK, edges, an inflation and sampling on
a one-joint arm whose answers follow from its geometry."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "csdecomp_b200")


def build(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libcsdecomp_b200.so")):
        pytest.skip("libcsdecomp_b200.so is not built")
    exe = str(tmp_path / "adapter_demo")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "adapter_demo.cpp"), "-L", LIBDIR, "-lcsdecomp_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_adapter_compiles_and_maps_errors(tmp_path):
    exe = build(tmp_path)
    import torch
    if torch.cuda.is_available():
        pytest.skip("the no-device path needs a machine without a GPU")
    r = subprocess.run([exe, "nodevice"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")


@pytest.mark.gpu
def test_adapter_on_the_gpu(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe, "device"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok faces=")
