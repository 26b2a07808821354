"""Synthetic workload generators: shapes, sizes and non-overlapping starts."""
import numpy as np
from scipy.spatial import cKDTree

import gb2_scenarios as S


def no_overlap(a):
    x, r = a["x"], a["radius"]
    t = cKDTree(x)
    pairs = t.query_pairs(2 * r.max())
    for i, j in pairs:
        assert np.linalg.norm(x[i] - x[j]) >= r[i] + r[j]


def test_sphere_pour_shape():
    sc = S.sphere_pour()
    a = sc["atoms"]
    assert len(a["tag"]) == 20000 and np.all(a["radius"] == 1e-3)
    assert a["x"][:, 2].min() > 1e-3 and a["x"][:, 2].max() < 0.2
    assert np.all(np.abs(a["v"]) <= 0.1)
    no_overlap(S.subset(sc, 3000)["atoms"])


def test_hopper_shape():
    sc = S.hopper(n=20000, gap=0.01, vmax=0.05)
    a = sc["atoms"]
    assert a["radius"].min() >= 0.5e-3 and a["radius"].max() <= 2e-3
    assert abs(np.median(S.hopper(n=200000)["atoms"]["radius"]) - 1e-3) < 2e-5
    no_overlap(a)
    nodes = sc["fixes"][1]["nodes"]
    assert nodes.shape == (8192, 3, 3)
    for d in range(3):
        assert nodes[:, :, d].min() > sc["boxlo"][d] and nodes[:, :, d].max() < sc["boxhi"][d]
