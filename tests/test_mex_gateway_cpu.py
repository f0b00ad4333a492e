"""The MEX gateway compiles against the C ABI (a syntax and type check with a declarations-only
mex.h stand-in; MATLAB's own mex.h is not in this image)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_gateway_compiles_against_the_c_abi():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "tests", "mexstub"),
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "petakit5d_b200", "mex", "pkdecon_mex.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
