"""Superquadric path on the GPU against the superquadric oracle.

Bar: the contact-point solve is held to its own convergence tolerance, not
bit parity (non-integer blockiness goes through pow(), whose last bit
differs between CUDA's math library and the host's).  So the pair list and
the contact states must agree exactly, contact points to 1e-9 of the
particle size, and forces and torques to 1e-6 of the largest pair force;
after a short run, positions and velocities agree to the same level.
"""
import numpy as np
import pytest

import gb2_scenarios as S
import oracle

pytestmark = pytest.mark.gpu


def _pair(n=343, seed=3, fill=0.8):
    import granb200
    sc = S.sq_packing(n=n, seed=seed, fill=fill)
    return sc, granb200.SqEngine(sc), oracle.SqOracle(sc)


def _cmp_pairs(e, o, size):
    p, q = e.pairs(), o.pairs()
    assert np.array_equal(p["tag_i"], q["tag_i"]) and np.array_equal(p["tag_j"], q["tag_j"]), "pair lists differ"
    assert np.array_equal(p["state"], q["state"]), "contact states differ at %d pairs" % int((p["state"] != q["state"]).sum())
    live = q["state"] > 0
    d = np.abs(p["cp"][live] - q["cp"][live]).max() if live.any() else 0.0
    assert d <= 1e-9 * size, "contact points differ by %.3g m" % d
    return int((q["state"] == 2).sum())


def _cmp_forces(e, o, rtol=1e-6):
    a, b = e.atoms(), o.atoms()
    fs = np.abs(b["f"]).max()
    ts = np.abs(b["torque"]).max()
    df = np.abs(a["f"] - b["f"]).max()
    dt = np.abs(a["torque"] - b["torque"]).max()
    assert df <= rtol * fs, "force error %.3g of max %.3g" % (df, fs)
    assert dt <= rtol * ts, "torque error %.3g of max %.3g" % (dt, ts)
    return a, b


def test_sq_setup_matches_oracle():
    sc, e, o = _pair()
    e.setup()
    o.setup()
    nint = _cmp_pairs(e, o, 1e-3)
    assert nint > 0
    _cmp_forces(e, o)


def test_sq_run_matches_oracle():
    sc, e, o = _pair()
    e.setup()
    o.setup()
    total = 0
    for _ in range(3):
        e.run(100)
        o.run(100)
        total += _cmp_pairs(e, o, 1e-3)
        a, b = _cmp_forces(e, o, rtol=1e-5)
        assert np.abs(a["x"] - b["x"]).max() <= 1e-12
        assert np.abs(a["v"] - b["v"]).max() <= 1e-8 * np.abs(b["v"]).max()
        assert np.abs(a["quat"] - b["quat"]).max() <= 1e-9
    assert total > 0
    ce, co = e.counters(), o.counters()
    assert ce["nbuilds"] == co["nbuilds"]
    assert ce["pairs_solved"] == co["pairs_solved"]
    assert abs(ce["iters"] - co["iters"]) <= 0.01 * co["iters"]


def test_sq_free_rotation_matches_oracle():
    """One torque-free particle: the integrator alone (no contact), 2000 steps."""
    import granb200
    rng = np.random.default_rng(9)
    shape = np.array([[2e-3, 1.2e-3, 1e-3]])
    blk = np.array([3.5])
    vol = S.sq_volume(shape, blk)
    sc = {"dt": 1e-5, "skin": 5e-4, "youngs": 5e6, "poisson": 0.45, "restitution": 0.3, "friction": 0.5,
          "atoms": {"x": np.zeros((1, 3)), "v": np.array([[0.1, 0.0, 0.0]]), "quat": S.random_quaternions(rng, 1),
                    "angmom": np.array([[3e-9, -2e-9, 4e-9]]), "shape": shape, "blockiness": blk,
                    "rmass": vol * 2500.0, "inertia": S.sq_inertia(shape, blk, 2500.0), "volume": vol}}
    e, o = granb200.SqEngine(sc), oracle.SqOracle(sc)
    e.setup()
    o.setup()
    e.run(2000)
    o.run(2000)
    a, b = e.atoms(), o.atoms()
    for k in ("quat", "angmom", "omega", "x"):
        assert np.allclose(a[k], b[k], rtol=1e-12, atol=1e-15), k
