"""The C++ host adapter (include/tsp_b200_backend.hpp) drives the backend like the reference's
SimulationMgr drives I_SimBackend: compiled with g++ against the C ABI and run on the GPU."""
import os
import subprocess

import pytest

from turbospharticles_b200 import abi

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_adapter_free_fall(tmp_path):
    exe = str(tmp_path / "adapter_step")
    lib_dir = os.path.dirname(abi.LIB_PATH)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "adapter_step.cpp"), "-L", lib_dir, "-ltsp_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dy=" in r.stdout
