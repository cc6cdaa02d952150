"""The host SAH BLAS builder (vork_b200/csrc/vkb_sah.h) builds the same tree on one
thread and on every hardware thread (subtrees spliced in depth-first order), no GPU."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CUDA_INC = Path("/usr/local/cuda/include")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx or not (CUDA_INC / "vector_types.h").exists():
        pytest.skip("needs g++ and the CUDA headers")
    exe = tmp_path_factory.mktemp("sah") / "sah_harness"
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", f"-I{ROOT / 'vork_b200' / 'csrc'}", f"-I{CUDA_INC}",
                    str(ROOT / "tests" / "sah_harness.cpp"), "-o", str(exe)], check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("grid,soup", [(0, 3), (20, 0), (400, 60000)])
def test_threaded_build_equals_one_thread_build(harness, grid, soup):
    r = subprocess.run([str(harness), str(grid), str(soup)], capture_output=True, text=True, timeout=300)
    print(r.stdout.strip())
    assert r.returncode == 0 and r.stdout.startswith("SAME"), r.stdout + r.stderr
