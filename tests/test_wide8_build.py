"""The host collapse into compressed 8-wide BLAS nodes (vork_b200/csrc/vkb_wide8.h), no GPU:
the leaf order is a permutation, every used slot's decoded box holds every triangle under
it, and closest hits through the wide tree equal a brute-force test of every triangle."""
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
    exe = tmp_path_factory.mktemp("wide8") / "wide8_harness"
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", f"-I{ROOT / 'vork_b200' / 'csrc'}", f"-I{CUDA_INC}",
                    str(ROOT / "tests" / "wide8_harness.cpp"), "-o", str(exe)], check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("grid,soup,rays", [(0, 1, 50), (0, 9, 300), (60, 3000, 3000), (300, 40000, 600)])
def test_wide8_collapse_is_exact_and_conservative(harness, grid, soup, rays):
    r = subprocess.run([str(harness), str(grid), str(soup), str(rays)], capture_output=True, text=True, timeout=300)
    print(r.stdout.strip())
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
