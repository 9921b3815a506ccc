"""The 8-wide scene-BVH builder (speedball_b200/csrc/sb_flat_build.cpp) on the
CPU: compiled with g++ beside tests/native/wide_build_check.cpp and run on
random boxes with random instance slots, including a scene small enough to be
a single leaf. Every item once, inside its leaf slot's box, leaves of 1..3
items in slot order, children after their parents, depth as reported."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    exe = tmp_path_factory.mktemp("wide") / "wide_build_check"
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", str(ROOT / "speedball_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "wide_build_check.cpp"),
                    str(ROOT / "speedball_b200" / "csrc" / "sb_flat_build.cpp"), "-o", str(exe), "-lpthread"],
                   check=True)
    return exe


@pytest.mark.parametrize("n,seed", [(1, 1), (3, 2), (40, 3), (50_000, 4), (200_000, 5)])
def test_wide_tree_covers_every_item(checker, n, seed):
    r = subprocess.run([str(checker), str(n), str(seed)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
