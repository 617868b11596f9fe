"""The C++ drop-in headers (include/shockhash_b200/ShockHash.h, ShockHash2.h, ShockHash2Flat.h, SIMDShockHash.h)
compiled into the reference's README example (README.md:41-47) and linked against libshg.so."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "shockhash_b200", "_lib")
SRC = os.path.join(ROOT, "tests", "cpp", "readme_dropin.cpp")


def _compile(out, std):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libshg.so")):
        pytest.skip("libshg.so not built")
    cmd = ["g++", f"-std={std}", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + LIBDIR, "-lshg", "-Wl,-rpath," + LIBDIR, "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.parametrize("std", ["c++17", "c++20"])
def test_dropin_headers_compile_and_link(tmp_path, std):
    _compile(str(tmp_path / "readme"), std)


@pytest.mark.gpu
def test_dropin_readme_example(tmp_path):
    exe = str(tmp_path / "readme")
    _compile(exe, "c++20")
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=300).stdout.splitlines()
    assert out[0].split() == ["1", "3", "2", "0"]
    assert out[1].startswith("ShockHash2 ok")
    assert float(out[1].split()[2]) < 2.0
    assert out[2] == "ShockHash2Flat ok"
    assert out[3] == "ShockHash hash128 ok"
    assert out[4] == "ShockHash rotation ok"
    assert out[5] == "SIMDShockHash ok"
