"""The C++ drop-in: a driver written against the reference's classes compiles
against include/mmprop with only the header and class name changed, and on a
GPU reproduces the reference's own output (tests/golden/dropin_two_mode.npz,
made by building the same driver against the reference sources)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DRIVER = os.path.join(ROOT, "tests", "dropin", "two_mode_driver.cpp")
LIBDIR = os.path.join(ROOT, "mm_propagation_b200")


def build(tmp_path):
    exe = str(tmp_path / "two_mode_b200")
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-Wall", "-Werror",
                    "-I" + os.path.join(ROOT, "include", "mmprop"), "-I" + os.path.join(ROOT, "include"),
                    DRIVER, "-o", exe, "-L" + LIBDIR, "-lmmp_b200", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def test_driver_compiles_against_dropin_headers(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_driver_matches_reference_output(tmp_path):
    exe = build(tmp_path)
    out = tmp_path / "out.txt"
    subprocess.run([exe, str(out)], check=True)
    a = np.loadtxt(out)
    phi = (a[:, 0] + 1j * a[:, 1]).reshape(2, -1)
    ref = np.load(os.path.join(ROOT, "tests", "golden", "dropin_two_mode.npz"))["result"]
    err = np.sqrt((np.abs(phi - ref) ** 2).sum(-1) / (np.abs(ref) ** 2).sum(-1)).max()
    assert err < 1e-5, err   # default FP32-bulk arithmetic
