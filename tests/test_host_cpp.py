"""The C++ MpmSim API header (mpmsnow_b200/host/MpmSim.h) without a GPU: the reference-style test program
compiles with warnings as errors, links against the library, and reports the missing device through the
library's status (the GPU run is tests/test_gpu_host_cpp.py)."""
import subprocess

import pytest

from tests.host_cpp.build import build_test_program


def test_header_compiles_links_and_reports_no_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: tests/test_gpu_host_cpp.py runs the program")
    exe = build_test_program(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("NO_DEVICE")


def test_sop_header_compiles_links_and_reports_no_device(tmp_path):
    """The Houdini SOP's cook logic over the C++ API (mpmsnow_b200/host/MpmSimSOP.h, tests/host_cpp/test_sop.cpp)
    compiles with warnings as errors and links; without a device the seeding reports it."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: tests/test_gpu_host_cpp.py runs the program")
    exe = build_test_program(tmp_path, "test_sop")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3 and r.stdout.startswith("NO_DEVICE"), (r.returncode, r.stdout, r.stderr)


def test_header_host_logic(tmp_path):
    """Descriptors, set ownership, termination parameters and the arguments Sim rejects before any device call
    (tests/host_cpp/test_descriptors.cpp); runs with or without a device."""
    exe = build_test_program(tmp_path, "test_descriptors")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "OK", (r.returncode, r.stdout, r.stderr)

