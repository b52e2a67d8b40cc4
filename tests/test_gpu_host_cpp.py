"""The C++ MpmSim API (mpmsnow_b200/host/MpmSim.h) on a B200, through the reference-style test program
tests/host_cpp/test_mpmsim.cpp: body partition, the gravity known answer (TestSimClass.cpp:120-190), particle
variables and uploads, the unknown-variable message, cancellation and the Debug hook."""
import subprocess

import pytest

from tests.host_cpp.build import build_test_program

pytestmark = pytest.mark.gpu


def test_cpp_api_program(tmp_path):
    exe = build_test_program(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), (r.returncode, r.stdout, r.stderr)


def test_sop_cook_program(tmp_path):
    """The Houdini SOP's cook logic (mpmsnow_b200/host/MpmSimSOP.h) on a B200: GPU seeding from a sampled SDF
    bit-identical to a host restatement of SOP_MPMSim.cpp:168-214, cooks with a sampled ground, an interrupted
    cook (tests/host_cpp/test_sop.cpp)."""
    exe = build_test_program(tmp_path, "test_sop")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), (r.returncode, r.stdout, r.stderr)
