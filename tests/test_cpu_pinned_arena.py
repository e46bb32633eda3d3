"""The continuous-batching service's pinned output arena (csrc/pinned_arena.h), built for
the host with malloc standing in for page-locking: pieces never overlap and are aligned,
a stream of mixed picture sizes stops growing the arena once it covers the peak held at
once, and released pieces merge back into whole chunks."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_pinned_arena(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "pinned_arena_test")
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", "-o", exe,
                    os.path.join(ROOT, "tests", "pinned_arena_test.cpp")], check=True)
    r = subprocess.run([exe], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout
