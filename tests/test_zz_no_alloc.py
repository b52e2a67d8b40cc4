"""The no-allocation body segmentation entry point, through the C-ABI — needs a B200.

mpm_calculate_bodies_noalloc serves callers that cannot allocate device memory when they need the body
partition (graph capture, hosts that own the GPU's memory, latency-critical paths): it works in a fixed device
array inside the library.  This file is collected last so that a run stopping at the first failure has run
every other test first; it passes alone in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cloud_and_bodies(seed, n):
    """A cloud with many bodies and singletons, plus the body partition the allocating path computes for it
    (mpm_create runs Sim::calculateBodies; mpm_get_bodies returns it), checked against the oracle's."""
    from mpmsnow_b200 import scenes as S
    from mpmsnow_b200 import sim as M
    rng = np.random.default_rng(seed)
    cloud = rng.uniform(0, 0.35, (n - 2000, 3)).astype(np.float32)
    ball = S.sphere_points(2000, 0.05, (0.5, 0.5, 0.5), seed + 1)
    x = np.concatenate([cloud, ball]).astype(np.float32)
    h = 0.012
    sim = M.Sim(x, np.ones(n, dtype=np.float32), h, M.CubicBsplineShapeFunction(),
                M.SnowConstitutiveModel(*S.SNOW), M.CollisionObjectSet(), M.ForceFieldSet())
    body, nb, nbal = sim.bodies()
    # the oracle's Sim::calculateBodies (exact radius query in place of the KD-tree) on the same cloud
    from oracle import oracle as O
    O.build()
    o = O.OracleSim(x, np.ones(n, dtype=np.float32), h, S.SNOW, [], [], prec=32)
    ob, onb, onbal = o.bodies()
    assert np.array_equal(ob, body) and (onb, onbal) == (nb, nbal)
    return x, h, body, nb, nbal


def test_noalloc_bodies_match_the_allocating_path_and_the_oracle():
    import torch

    from mpmsnow_b200 import build, capi
    build.build()
    L = capi.load()
    assert L.mpm_calculate_bodies_noalloc_max() == 262144
    torch.cuda.init()
    stream = torch.cuda.current_stream().cuda_stream
    for call, (seed, n) in enumerate([(41, 20000), (42, 15000)]):   # two calls in a row
        x, h, body_ref, nb, nbal = _cloud_and_bodies(seed, n)
        assert nb > 10 and nbal > 10
        x_dev = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()          # component-major
        body_dev = torch.full((n,), 12345, dtype=torch.int32, device="cuda")
        counts_dev = torch.full((2,), -7, dtype=torch.int32, device="cuda")
        rc = L.mpm_calculate_bodies_noalloc(x_dev.data_ptr(), n, h, body_dev.data_ptr(), counts_dev.data_ptr(),
                                            C.c_void_p(stream))
        assert rc == 0, capi.STATUS.get(rc, rc)
        torch.cuda.synchronize()
        assert np.array_equal(body_dev.cpu().numpy(), body_ref), call
        assert counts_dev.cpu().tolist() == [nb, nbal], call


def test_noalloc_rejects_more_than_its_maximum():
    import torch

    from mpmsnow_b200 import build, capi
    build.build()
    L = capi.load()
    n = L.mpm_calculate_bodies_noalloc_max() + 1
    x_dev = torch.zeros(3 * 4, dtype=torch.float32, device="cuda")
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = L.mpm_calculate_bodies_noalloc(x_dev.data_ptr(), n, 0.01, out.data_ptr(), out.data_ptr(), None)
    assert rc == 17  # MPM_ERR_TOO_MANY_PARTICLES, rejected before any device work
    assert "maximum" in L.mpm_status_string(rc).decode()
