"""The C++17 drop-in (include/pt_cuda_renderer.hpp) driven by the reference's own code.

oracle/_ref/dropin_check is built from oracle/dropin_check.cpp against the reference's headers
and its src/cuda/cuda_renderer.cu: it builds a scene with the reference's classes (spheres,
bvh_node, materials, camera, flatten_scene) and renders and queries it through the reference's
cuda_renderer / cuda_query_rays and through ptb::cuda_renderer / ptb::cuda_query_rays, passing the
reference's own flat_scene, flat_camera, ray and trace_result types.  It exits 0 when every image
(all six debug views, MIS and classic lighting), ray count, RGBA buffer and query record agrees
bit for bit, and checks that invalid dimensions raise std::invalid_argument.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
DROPIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "dropin_check"


@pytest.mark.skipif(not DROPIN.exists(), reason="oracle/_ref/dropin_check is not built")
def test_reference_types_through_the_cpp_dropin_are_bit_identical():
    run = subprocess.run([str(DROPIN)], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout + run.stderr
    lines = run.stdout.splitlines()
    assert sum("identical" in l for l in lines) == 6 * 2 + 2, run.stdout
    assert "invalid dimensions rejected: yes" in run.stdout
