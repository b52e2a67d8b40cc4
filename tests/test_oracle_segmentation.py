"""The oracle's body segmentation (Sim::calculateBodies, Sim.cpp:136-203, with the KD-tree's strict radius
query, KdTree.inl:186-191) against connected components computed independently here: every pair whose FP32
squared distance, summed as (dx² + dy²) + dz², is below h², by scipy's graph components.  Bodies are numbered
in the order of their smallest particle index and one-particle components are ballistic (-1), as the
reference's flood fill from each unprocessed particle in index order numbers them.  The GPU partition tests
compare the CUDA segmentation with this oracle bit for bit, so this pins what they compare against."""
import numpy as np
import pytest
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components
from scipy.spatial import cKDTree

from mpmsnow_b200 import scenes as S


def brute_bodies(x, h):
    x = np.asarray(x, dtype=np.float32)
    n = x.shape[0]
    h32 = np.float32(h)
    pairs = cKDTree(x.astype(np.float64)).query_pairs(float(h) * 1.001, output_type="ndarray")
    if len(pairs):
        d = x[pairs[:, 0]] - x[pairs[:, 1]]
        s = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        pairs = pairs[s < h32 * h32]
    g = coo_matrix((np.ones(len(pairs)), (pairs[:, 0], pairs[:, 1])), shape=(n, n)) if len(pairs) else \
        coo_matrix((n, n))
    _, comp = connected_components(g, directed=False)
    size = np.bincount(comp)
    first = np.full(size.shape[0], n, dtype=np.int64)
    np.minimum.at(first, comp, np.arange(n))
    order = np.argsort(first[size >= 2])
    label_of = np.full(size.shape[0], -1, dtype=np.int64)
    label_of[np.nonzero(size >= 2)[0][order]] = np.arange(order.shape[0])
    body = label_of[comp].astype(np.int32)
    return body, int((size >= 2).sum()), int((size == 1).sum())


def oracle_bodies(x, h):
    from oracle import oracle as O
    O.build()
    n = x.shape[0]
    sim = O.OracleSim(x, np.ones(n, dtype=np.float32), h, S.SNOW, [], [], prec=32)
    return sim.bodies()


@pytest.mark.parametrize("seed,n,extent,h", [(1, 3000, 0.3, 0.012), (2, 5000, 0.2, 0.012), (3, 2000, 1.0, 0.05),
                                             (4, 4000, 0.5, 0.02)])
def test_oracle_bodies_match_brute_force_components(seed, n, extent, h):
    x = np.random.default_rng(seed).uniform(0, extent, (n, 3)).astype(np.float32)
    b_o, nb_o, nbal_o = oracle_bodies(x, h)
    b_r, nb_r, nbal_r = brute_bodies(x, h)
    assert nb_o > 50 and nbal_o > 50  # many bodies and singletons in every cloud
    assert (nb_o, nbal_o) == (nb_r, nbal_r)
    assert np.array_equal(b_o, b_r)


def test_oracle_bodies_strict_radius_on_a_lattice():
    """Lattice points exactly one spacing apart: with the spacing at h (after FP32 rounding of the coordinates)
    only pairs whose FP32 squared distance falls below h² link, which the independent predicate reproduces."""
    h = 0.1
    g = np.arange(12, dtype=np.float32) * np.float32(h)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], 1).astype(np.float32)
    x = np.concatenate([x, x[:200] + np.float32(0.03)])  # a few particles closer than h to lattice points
    b_o, nb_o, nbal_o = oracle_bodies(x, h)
    b_r, nb_r, nbal_r = brute_bodies(x, h)
    assert nb_o > 100 and nbal_o > 10  # some lattice neighbours round below h, most do not
    assert (nb_o, nbal_o) == (nb_r, nbal_r)
    assert np.array_equal(b_o, b_r)
