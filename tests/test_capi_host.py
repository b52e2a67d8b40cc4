"""Host-side checks of the C-ABI library that need no GPU: it builds, loads, exports every entry point that
include/mpm_gpu.h declares, and its host logic reports errors instead of falling back to the CPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from mpmsnow_b200 import build, capi
    build.build()
    return capi.load()


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "mpm_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mpm_[a-z0-9_]+)\s*\(", src)) - {"mpm_cancel_fn", "mpm_iterate_fn"})


def test_every_declared_symbol_is_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "mpmsnow_b200", "libmpmsnow_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (mpm_\w+)", out))
    decl = declared_symbols()
    assert len(decl) >= 18
    missing = [s for s in decl if s not in exported]
    assert not missing, missing
    from mpmsnow_b200 import capi
    assert sorted(capi.EXPORTS) == decl


def test_library_targets_sm100a(lib):
    from mpmsnow_b200 import build
    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags and "fast-math" not in flags


def test_status_strings_carry_reference_messages(lib):
    assert lib.mpm_abi_version() == 2
    assert lib.mpm_status_string(9).decode() == "nans in particle velocity data!"
    assert lib.mpm_status_string(10).decode() == "grid is too big"
    assert lib.mpm_status_string(4).decode() == "nans in splatted masses!"


def test_invalid_arguments_rejected_before_touching_a_device(lib):
    from mpmsnow_b200 import capi
    d = capi.MpmSceneDesc()
    d.grid_size = 0.01
    d.dimension = 4
    d.shape_function = 0
    h = C.c_void_p()
    x = np.zeros(3, dtype=np.float32)
    m = np.ones(1, dtype=np.float32)
    assert lib.mpm_create(C.byref(d), 1, x, m, C.byref(h)) == 13   # no 4-D grids: MPM_ERR_UNSUPPORTED
    d.dimension = 0
    assert lib.mpm_create(C.byref(d), 1, x, m, C.byref(h)) == 13
    d.dimension = 3
    d.num_colliders = 99
    assert lib.mpm_create(C.byref(d), 1, x, m, C.byref(h)) == 13
    d.num_colliders = 0
    d.grid_size = 0.0
    assert lib.mpm_create(C.byref(d), 1, x, m, C.byref(h)) == 1    # MPM_ERR_INVALID_ARGUMENT


def test_no_cpu_fallback_without_a_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from mpmsnow_b200 import capi
    d = capi.MpmSceneDesc()
    d.grid_size = 0.01
    d.dimension = 3
    d.youngs_modulus = 1.4e5
    d.poisson_ratio = 0.2
    h = C.c_void_p()
    x = np.zeros(3, dtype=np.float32)
    m = np.ones(1, dtype=np.float32)
    assert lib.mpm_create(C.byref(d), 1, x, m, C.byref(h)) == 3    # MPM_ERR_NO_DEVICE


def test_scene_shapes():
    from mpmsnow_b200 import scenes as S
    c1 = S.snowball()
    assert c1["x"].shape == (10000, 3) and c1["h"] == 0.01 and c1["dt"] == 5e-4
    r = np.linalg.norm(c1["x"] - np.float32([0, 0.3, 0]), axis=1)
    assert r.max() < 0.1
    assert abs(c1["m"].sum() - 400 * 4 / 3 * np.pi * 0.1 ** 3) < 1e-4
    c3 = S.slab(cells=(17, 4, 9))
    assert c3["x"].shape[0] == 8 * 17 * 4 * 9
    assert 1e5 / 2.4 * 0.999 < c3["mu0"].min() and c3["mu0"].max() < 2e5 / 2.4 * 1.001
    a = np.radians(30)
    phi = -np.sin(a) * c3["x"][:, 0] + np.cos(a) * c3["x"][:, 1]
    assert phi.min() > 0   # the slab starts above its plane
