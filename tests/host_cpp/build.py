"""Compile the C++ test programs in tests/host_cpp against the C++ MpmSim header and the in-tree library."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def build_test_program(out_dir, name="test_mpmsim"):
    """Compile tests/host_cpp/<name>.cpp with warnings as errors; returns the executable's path."""
    from mpmsnow_b200 import build
    build.build()
    pkg = os.path.join(ROOT, "mpmsnow_b200")
    exe = os.path.join(str(out_dir), name)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(pkg, "host"), os.path.join(ROOT, "tests", "host_cpp", name + ".cpp"),
           "-L", pkg, "-lmpmsnow_b200", f"-Wl,-rpath,{pkg}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
