"""The ray_tracer command line (cuda-path-tracer_b200/cli/ray_tracer.cpp) without a GPU: the
argument checks of the reference's render_tests.py (tests/render_tests.py:27-31: exit 1, nothing
on stdout), --help, and exit 77 when no CUDA device is usable."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

import ptb200 as pt

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "cuda-path-tracer_b200" / "ray_tracer"
pytestmark = pytest.mark.skipif(not CLI.exists(), reason="ray_tracer not built (make -C cuda-path-tracer_b200)")


def run(*args, timeout=30):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, timeout=timeout)


def test_help():
    r = run("--help")
    assert r.returncode == 0
    for flag in ("--obj FILE", "--width N", "--batch-samples N", "--obj-rotate X Y Z", "--lighting classic|mis",
                 "shaded|normals|triangle-id|material-id|bvh|intersections"):
        assert flag.encode() in r.stdout


@pytest.mark.parametrize("args, message", [
    (["--backend", "reference"], "CUDA is the only rendering backend"),
    (["--backend", "portable-brute"], "CUDA is the only rendering backend"),
    (["--samples", "0"], "invalid integer: 0"),
    (["--width", "0"], "invalid integer: 0"),
    (["--height", "x"], "invalid integer: x"),
    (["--seed", "-1"], "invalid integer: -1"),
    (["--obj"], "missing value for --obj"),
    (["--debug", "invalid"], "unknown debug mode: invalid"),
    (["--lighting", "invalid"], "lighting must be classic or mis"),
    (["--cuda-block", "3", "3"], "unknown option: --cuda-block"),
    (["--obj-scale", "1", "2"], "expected three values for --obj-scale"),
    (["--obj-rotate", "0", "90", "0"], "OBJ transforms require --obj FILE"),
    (["--obj", "x.obj", "--obj-scale", "1", "0", "1"], "nonzero scale"),
    (["--obj", "x.obj", "--obj-translate", "1", "nan", "1"], "invalid finite number: nan"),
    (["--obj", ""], "OBJ filename must not be empty"),
])
def test_argument_errors(args, message):
    r = run(*args)
    assert r.returncode == 1 and not r.stdout
    assert message.encode() in r.stderr and b"Use --help for usage." in r.stderr


def test_no_device_exits_77():
    available, _ = pt.cuda_device_available()
    if available:
        pytest.skip("a CUDA device is present")
    r = run("--obj", ROOT / "tests" / "golden" / "obj" / "fixture.obj", "--samples", "1")
    assert r.returncode == 77 and not r.stdout
    assert r.stderr.startswith(b"CUDA device unavailable:")
