"""The body segmentation's scheme, restated sequentially on the CPU with random processing orders (the CUDA
passes in mpmsnow_b200/csrc/mpm_kernels.cu run their unions in whatever order the GPU schedules them):
  - the first segmentation joins sampled close pairs, then every particle outside the giant component joins
    all its close neighbours (k_seg_sample, k_seg_giant, k_seg_finish);
  - every union that hooks a root records the pair that caused it (uf_union), so one segmentation's pairs
    are a spanning forest of its components: N - components pairs;
  - a later segmentation re-checks the last forest's pairs against the current positions (k_seg_links) in
    place of the sample, and the finish pass makes it exact whatever pairs survived.
Between segmentations the particles move and are permuted into a new slot order; the forest is kept by caller
index and found again through slotOf, as in the step.  Every partition is compared with connected components
computed independently (test_oracle_segmentation.brute_bodies).  The CUDA kernels themselves are compared with
the oracle on the GPU (tests/test_gpu_parity.py)."""
import numpy as np

from tests.test_oracle_segmentation import brute_bodies


def _close(x, i, j, h2):
    d = x[i] - x[j]
    return (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2] < h2


def _find(parent, a):
    while parent[a] != a:
        parent[a] = parent[parent[a]]
        a = parent[a]
    return a


def _union(parent, i, j, rec, orig):
    a, b = _find(parent, i), _find(parent, j)
    if a == b:
        return
    if a > b:
        a, b = b, a
    parent[b] = a
    rec[b] = (orig[i], orig[j])


def _segment(x, h, orig, slot_of, forest, nbrs, rng):
    n = x.shape[0]
    h2 = np.float32(h) * np.float32(h)
    parent = list(range(n))
    rec = np.full((n, 2), -1, dtype=np.int64)
    if forest is None:
        for i in rng.permutation(n):
            for j in nbrs[i][:3]:
                _union(parent, i, j, rec, orig)
    else:
        for k in rng.permutation(n):
            a, c = forest[k]
            if a >= 0 and _close(x, slot_of[a], slot_of[c], h2):
                _union(parent, slot_of[a], slot_of[c], rec, orig)
    roots, counts = np.unique([_find(parent, i) for i in range(n)], return_counts=True)
    giant = roots[np.argmax(counts)]
    outside = 0
    for i in rng.permutation(n):
        if _find(parent, i) == _find(parent, giant):
            continue
        outside += 1
        for j in nbrs[i]:
            _union(parent, i, j, rec, orig)
    root = np.array([_find(parent, i) for i in range(n)])
    return root, rec, outside


def _labels_by_caller(root, orig):
    """Bodies numbered by their smallest caller index, one-particle components -1, in caller order."""
    n = root.shape[0]
    size = np.bincount(root, minlength=n)
    first = np.full(n, n, dtype=np.int64)
    np.minimum.at(first, root, orig)
    body_roots = np.nonzero(size >= 2)[0]
    rank = np.full(n, -1, dtype=np.int64)
    rank[body_roots[np.argsort(first[body_roots])]] = np.arange(body_roots.shape[0])
    out = np.empty(n, dtype=np.int64)
    out[orig] = rank[root]
    return out


def _neighbours(x, h):
    from scipy.spatial import cKDTree
    h2 = np.float32(h) * np.float32(h)
    nb = [[] for _ in range(x.shape[0])]
    for i, j in cKDTree(x.astype(np.float64)).query_pairs(float(h) * 1.001):
        if _close(x, i, j, h2):
            nb[i].append(j)
            nb[j].append(i)
    return nb


def _run(x_caller, h, moves, rng):
    """Segment, then move and re-slot the particles and segment again from the recorded forest, len(moves)
    times; returns the outside-giant counts and checks every partition and forest."""
    n = x_caller.shape[0]
    orig = np.arange(n)
    forest = None
    outside_counts = []
    x_c = x_caller.astype(np.float32)
    for step in range(len(moves) + 1):
        if step > 0:
            x_c = (x_c + moves[step - 1]).astype(np.float32)
            orig = rng.permutation(n)          # the step's new slot order: slot s holds caller orig[s]
        slot_of = np.empty(n, dtype=np.int64)
        slot_of[orig] = np.arange(n)
        x = x_c[orig]
        root, rec, outside = _segment(x, h, orig, slot_of, forest, _neighbours(x, h), rng)
        body, nb, nbal = brute_bodies(x_c, h)
        assert np.array_equal(_labels_by_caller(root, orig), body), step
        assert int((rec[:, 0] >= 0).sum()) == n - np.unique(root).shape[0]  # a spanning forest
        forest = rec
        outside_counts.append(outside)
    return outside_counts


def test_forest_scheme_exact_on_a_cloud_that_joins_and_splits():
    rng = np.random.default_rng(5)
    n, h = 2500, 0.012
    x = rng.uniform(0, 0.15, (n, 3))
    moves = [np.zeros((n, 3)), rng.normal(0, 0.2 * h, (n, 3)), rng.normal(0, 1.0 * h, (n, 3)),
             np.where(x[:, :1] > 0.075, 0.05, 0.0) * np.array([[1.0, 0.0, 0.0]])]
    _run(x, h, moves, rng)


def test_forest_scheme_rebuilds_a_moving_body_without_search():
    """A dense body (2 particles per h along each axis, jittered) moving a little between segmentations: the
    forest's pairs hold, so almost every particle ends in the giant component without a neighbour search."""
    rng = np.random.default_rng(6)
    h = 0.02
    g = (np.arange(16) + 0.5) * (h / 2)
    X, Y, Z = np.meshgrid(g, g[:8], g[:10], indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + rng.uniform(-0.125, 0.125, (X.size, 3)) * h
    n = x.shape[0]
    moves = [np.full((n, 3), 0.003 * h) + rng.normal(0, 0.001 * h, (n, 3)) for _ in range(3)]
    outside = _run(x, h, moves, rng)
    assert outside[0] == 0 and max(outside[1:]) <= n // 50, outside
