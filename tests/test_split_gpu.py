"""Split precision (GB2_PREC_SPLIT) against the bit-exact FP64 path.

Split precision keeps positions, the overlap of every touching pair, walls,
gravity and the integration in FP64 and evaluates the sphere-sphere contact
chain in FP32 with Kahan-compensated FP32 per-atom sums.  The bar is a force
error within 1e-5 relative of FP64.  "Relative" is per atom and component
against the sum of the magnitudes of that atom's contributions (pair forces,
wall forces and weight), because the net force on a resting particle is a
near-cancelling sum and has no scale of its own:

    err_i = |f_split_i - f_fp64_i| / S_i,   S_i = sum_j |F_ij| + |f_i| + m_i g

Torques are held to the same bar with the lever arm r_i times S_i: a contact
torque is a contact radius times a tangential force bounded by the contact
force, and the tangential relative velocity at first contact is a
near-cancelling difference whose own relative error is not meaningful.

The FP64 engine is itself bit-identical to the oracle (test_parity_gpu.py),
so it serves as the FP64 reference here.
"""
import numpy as np
import pytest

import gb2_scenarios as S
import oracle
from parity_util import by_tag

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _engine(sc, split):
    import granb200
    return granb200.Engine(sc, precision=granb200.PREC_SPLIT if split else granb200.PREC_FP64)


def _state_scenario(sc, atoms):
    """Scenario whose atoms are a downloaded engine state (shear history starts at zero)."""
    out = dict(sc)
    a = dict(sc["atoms"])
    order = np.argsort(a["tag"])
    for k in ("radius", "rmass", "type", "tag"):
        a[k] = np.ascontiguousarray(a[k][order])
    b = by_tag(atoms)
    assert np.array_equal(b["tag"], a["tag"])
    for k in ("x", "v", "omega"):
        a[k] = np.ascontiguousarray(b[k])
    out["atoms"] = a
    return out


def _contribution_scale(sc, eng):
    """Per-atom force scale S_i: sum of |pair force| over touching pairs
    (oracle single-pair kernel on the engine's state and history), plus the
    net force and the weight; torque scale r_i S_i."""
    a = by_tag(eng.atoms())
    n = len(a["tag"])
    rad = np.zeros(n)
    mass = np.zeros(n)
    order = np.argsort(sc["atoms"]["tag"])
    rad[:] = sc["atoms"]["radius"][order]
    mass[:] = sc["atoms"]["rmass"][order]
    sf = mass * 9.81
    p = eng.pairs()
    for ti, tj, fl, h in zip(p["tag_i"], p["tag_j"], p["flag"], p["hist"]):
        i, j = ti - 1, tj - 1
        d = a["x"][i] - a["x"][j]
        if d @ d >= (rad[i] + rad[j]) ** 2:
            continue
        fi, tqi, fj, tqj, _ = oracle.pair_force(sc, a["x"][i], a["x"][j], a["v"][i], a["v"][j], a["omega"][i],
                                                a["omega"][j], rad[i], rad[j], mass[i], mass[j], shear=h.copy(),
                                                shearupdate=0)
        sf[i] += np.linalg.norm(fi)
        sf[j] += np.linalg.norm(fj)
    # wall contacts are FP64 in both precisions; the net force stands in for their scale
    sf += np.linalg.norm(a["f"], axis=1)
    return sf, rad * sf


def _errors(e64, e32, sf, st):
    a, b = by_tag(e64.atoms()), by_tag(e32.atoms())
    ef = np.max(np.abs(b["f"] - a["f"]), axis=1) / sf
    et = np.max(np.abs(b["torque"] - a["torque"]), axis=1) / st
    return ef, et


def _settled_hopper(n=6000, chunk=2000, max_steps=30000):
    """A small hopper after FP64 steps under gravity, run until at least n/2
    pairs touch, so the contact math is exercised on a compacted bed."""
    sc = S.hopper(n=n, seed=5, gap=0.002, vmax=0.2)
    e = _engine(sc, False)
    e.setup()
    done = 0
    while done < max_steps:
        e.run(chunk)
        done += chunk
        if e.census()["ntouch"] >= n // 2:
            break
    st = _state_scenario(sc, e.atoms())
    e.close()
    return st


def test_split_forces_at_setup():
    sc = _settled_hopper()
    e64, e32 = _engine(sc, False), _engine(sc, True)
    e64.setup()
    e32.setup()
    sf, st = _contribution_scale(sc, e64)
    ef, et = _errors(e64, e32, sf, st)
    ntouch = int((e64.pairs()["flag"] != 0).sum())
    assert ntouch >= 3000, "workload has too few contacts (%d) to test the contact math" % ntouch
    print("setup: touching pairs %d, max force err %.3g, max torque err %.3g" % (ntouch, ef.max(), et.max()))
    assert ef.max() <= TOL, "split force error %.3g > %g" % (ef.max(), TOL)
    assert et.max() <= TOL, "split torque error %.3g > %g" % (et.max(), TOL)


def test_split_forces_after_steps():
    """Same state, then a few steps in each precision with live shear history.

    The states drift apart by the split error itself, and a pair sitting on
    the Coulomb cap (|Ft| = mu |Fn|) may take the other branch in FP32, so the
    bound is on the 99.9th percentile, with a looser cap on the maximum."""
    sc = _settled_hopper()
    e64, e32 = _engine(sc, False), _engine(sc, True)
    e64.setup()
    e32.setup()
    e64.run(5)
    e32.run(5)
    sf, st = _contribution_scale(sc, e64)
    ef, et = _errors(e64, e32, sf, st)
    print("5 steps: p99.9 force err %.3g max %.3g; torque p99.9 %.3g max %.3g" % (
        np.quantile(ef, 0.999), ef.max(), np.quantile(et, 0.999), et.max()))
    assert np.quantile(ef, 0.999) <= TOL
    assert np.quantile(et, 0.999) <= TOL
    assert ef.max() <= 1e-3 and et.max() <= 1e-3
    # the pair set (same FP64 screening) and the neighbour lists agree exactly
    p, q = e64.pairs(), e32.pairs()
    assert np.array_equal(p["tag_i"], q["tag_i"]) and np.array_equal(p["tag_j"], q["tag_j"])
    assert np.array_equal(p["flag"], q["flag"])
    # shear history, as the tangential spring force kt |ds| it produces, on the same force bar
    a = by_tag(e64.atoms())
    rad = np.asarray(sc["atoms"]["radius"])[np.argsort(sc["atoms"]["tag"])]
    i, j = p["tag_i"] - 1, p["tag_j"] - 1
    dn = rad[i] + rad[j] - np.linalg.norm(a["x"][i] - a["x"][j], axis=1)
    reff = rad[i] * rad[j] / (rad[i] + rad[j])
    E, nu = sc["youngs"][0], sc["poisson"][0]
    geff = 1.0 / (2 * 2 * (2 - nu) * (1 + nu) / E)
    kt = 8.0 * geff * np.sqrt(reff * np.maximum(dn, 0.0))
    herr = kt * np.max(np.abs(p["hist"] - q["hist"]), axis=1) / np.minimum(sf[i], sf[j])
    print("5 steps: history error as force p99.9 %.3g max %.3g" % (np.quantile(herr, 0.999), herr.max()))
    assert np.quantile(herr, 0.999) <= TOL and herr.max() <= 1e-3


def _pour_stats(e, r, box):
    """Coordination number, packing fraction and cumulative overlap histogram."""
    a = e.atoms()
    p = e.pairs()
    x = by_tag(a)["x"]
    i, j = p["tag_i"] - 1, p["tag_j"] - 1
    d = x[i] - x[j]
    for k in (0, 1):   # periodic x/y minimum image
        d[:, k] -= box[k] * np.round(d[:, k] / box[k])
    ov = 2 * r - np.sqrt((d ** 2).sum(axis=1))
    touch = ov > 0
    z = np.sort(x[:, 2])
    top = z[int(0.98 * len(z))] + r
    phi = len(z) * 4.0 / 3.0 * np.pi * r ** 3 / (box[0] * box[1] * top)
    hist, _ = np.histogram(ov[touch] / r, bins=8, range=(0.0, 0.02))
    return np.array([2.0 * touch.sum() / len(x), phi]), np.cumsum(hist) / max(touch.sum(), 1)


def test_split_pour_statistics():
    """Sphere pour (80,000 spheres, config 1's pour on an 80 x 80 mm
    periodic floor) settled 0.8 s in each precision, then sampled 10 times
    over the next 0.2 s: the time-averaged coordination number, packing
    fraction and overlap distribution (cumulative histogram over 8 bins)
    agree within 1%.  Trajectories are chaotic, so only statistics compare;
    the spread between two FP64 realisations (another seed) is printed for
    reference.  The FP64 arm is the bit-exact path, pinned to the
    reference's own state digests on config 1's 20k pour and the other
    golden scenes, so its statistics stand for the reference's."""
    box = (0.08, 0.08, 0.2)
    res = []
    for split, seed in ((False, 12345), (True, 12345), (False, 777)):
        sc = S.sphere_pour(n=80000, seed=seed, box=box)
        e = _engine(sc, split)
        e.setup()
        e.run(80000)
        sa, ha = np.zeros(2), np.zeros(8)
        for _ in range(10):
            e.run(2000)
            st, h = _pour_stats(e, 1e-3, box)
            sa += st / 10
            ha += h / 10
        res.append((sa, ha))
        e.close()
    (a, ha), (b, hb), (c, hc) = res
    print("coordination %.4f / %.4f (other seed %.4f), packing %.4f / %.4f (%.4f)" % (a[0], b[0], c[0], a[1], b[1], c[1]))
    print("cumulative overlap histogram", np.round(ha, 4), np.round(hb, 4), "other seed", np.round(hc, 4))
    print("split vs fp64 %.4f, fp64 seed spread %.4f" % (np.abs(ha - hb).max(), np.abs(ha - hc).max()))
    assert abs(a[0] - b[0]) <= 0.01 * a[0]
    assert abs(a[1] - b[1]) <= 0.01 * a[1]
    assert np.abs(ha - hb).max() <= 0.01


def test_split_insert_pack():
    """fix insert/pack in split precision: insertion draws on the FP64 state,
    so the first insertion (before any step integrates) places exactly the
    FP64 path's particles; later ones follow the slightly different fill
    level of the region."""
    sc = S.insert_pour(insert_every=200)
    a, b = _engine(sc, True), _engine(sc, False)
    a.setup()
    b.setup()
    a.run(1)
    b.run(1)
    assert a.insert_stats() == b.insert_stats()
    xa, xb = by_tag(a.atoms()), by_tag(b.atoms())
    assert np.array_equal(xa["tag"], xb["tag"])
    new = xa["tag"] > len(sc["atoms"]["tag"])
    assert np.array_equal(xa["x"][new], xb["x"][new])
    a.run(600)
    b.run(600)
    sa, sb = a.insert_stats(), b.insert_stats()
    assert sa["next_step"] == sb["next_step"] == 801
    assert abs(sa["ninserted"] - sb["ninserted"]) <= 0.05 * sb["ninserted"]
