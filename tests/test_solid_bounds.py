"""The camera tracer skips the plane tests of a convex solid whose bounding
sphere a ray misses.  The sphere comes from `sc::solid_bound`
(spectral_b200/csrc/solid_bound.h, host code).  This CPU test compiles
tests/solid_bound_check.cpp against it with g++ and runs it.  It checks a
cube's exact sphere; unbounded solids (open box, half-space, slab, uncapped
prism, normals in one hemisphere) get no sphere; and every sampled point of
bounded solids (capped prism, tetrahedron, 180-odd random polytopes) lies
inside its sphere."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_solid_bound_holds_every_solid(tmp_path):
    exe = str(tmp_path / "solid_bound_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "spectral_b200", "csrc"),
                    os.path.join(ROOT, "tests", "solid_bound_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout
