"""Comparison helpers for engine-vs-oracle parity tests."""
import numpy as np

from granb200 import restart_scenario  # noqa: F401  (restart helper shared with the bench)


def by_tag(a):
    order = np.argsort(a["tag"])
    return {k: v[order] for k, v in a.items()}


def max_rel(a, b):
    """max |a-b| / max(|b|, tiny) over all components (0 when bitwise equal)."""
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), 1e-300)
    return float(np.max(d / s)) if d.size else 0.0


def assert_atoms_equal(eng, orc, keys=("x", "v", "omega", "f", "torque"), rtol=0.0):
    a, b = eng.atoms(), orc.atoms()
    assert np.array_equal(a["tag"], b["tag"]), "atom order differs from the oracle (sort/pbc semantics)"
    for k in keys:
        if rtol == 0.0:
            bad = np.argwhere(a[k] != b[k])
            assert bad.size == 0, "%s differs at %d entries, first atom tag %d: %r vs %r" % (
                k, len(bad), a["tag"][bad[0][0]], a[k][bad[0][0]], b[k][bad[0][0]])
        else:
            assert max_rel(a[k], b[k]) <= rtol, k


def assert_pairs_equal(eng, orc):
    p, q = eng.pairs(), orc.pairs()
    assert len(p["tag_i"]) == len(q["tag_i"]), "pair count %d vs %d" % (len(p["tag_i"]), len(q["tag_i"]))
    assert np.array_equal(p["tag_i"], q["tag_i"]) and np.array_equal(p["tag_j"], q["tag_j"]), "pair list differs"
    assert np.array_equal(p["flag"], q["flag"]), "contact flags differ"
    assert np.array_equal(p["hist"], q["hist"]), "shear history differs"
    return len(p["tag_i"]), int((q["flag"] != 0).sum())


def assert_mesh_equal(eng, orc, ifix):
    p, q = eng.mesh_contacts(ifix), orc.mesh_contacts(ifix)
    assert len(p["tag"]) == len(q["tag"]), "mesh contact count %d vs %d" % (len(p["tag"]), len(q["tag"]))
    assert np.array_equal(p["tag"], q["tag"]) and np.array_equal(p["tri"], q["tri"]), "mesh contact slots differ"
    assert np.array_equal(p["hist"], q["hist"]), "mesh shear history differs"
    return len(p["tag"])


def mesh_contact_map(mc):
    """{(tag, triangle): shear} of a mesh_contacts() download."""
    return {(int(t), int(r)): tuple(h) for t, r, h in zip(mc["tag"], mc["tri"], mc["hist"])}
