"""The C++ facade (static-pst-gpu.h) used the way the reference's testers use
StaticPSTGPU / StaticPSTGPUArr / intervalParallelSearch / formMetacellTags."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def test_cpp_facade_drop_in(tmp_path):
    pkg = ROOT / "static-priority-search-tree_b200"
    exe = tmp_path / "facade_drop_in"
    cmd = ["g++", "-std=c++20", "-O2", f"-I{ROOT / 'include'}", f"-I{pkg / 'cpp'}", "-I/usr/local/cuda/include",
           str(ROOT / "tests" / "cpp" / "facade_drop_in.cpp"), f"-L{pkg}", "-lpst_b200", "-L/usr/local/cuda/lib64",
           "-lcudart", f"-Wl,-rpath,{pkg}", "-o", str(exe)]
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "FACADE OK" in r.stdout, r.stdout + r.stderr
