"""Known-answer tests pinning the superquadric oracle (CPU only).

The superquadric contact path has no golden vectors in the reference, so the
oracle's restatement is pinned against analytic cases: spheres and aligned
ellipsoids through the superquadric solver, finite-difference derivatives of
the shape function, the optimality conditions of the converged contact
point, and the torque-free motion of the asphere integrator.
"""
import math

import numpy as np

import gb2_scenarios as S
import oracle


def _sphere_pair(r1, r2, gap):
    pa = {"center": [0.0, 0.0, 0.0], "quat": [1.0, 0.0, 0.0, 0.0], "shape": [r1] * 3, "n": 2.0}
    pb = {"center": [r1 + r2 + gap, 0.0, 0.0], "quat": [1.0, 0.0, 0.0, 0.0], "shape": [r2] * 3, "n": 2.0}
    return pa, pb


def test_sphere_contact_point_and_hertz_force():
    """Two spheres through the superquadric path: the pair force equals the
    sphere path's Hertz/history force for the same overlap and velocities."""
    r1, r2, ov = 1.0e-3, 1.5e-3, 2e-5
    sc = {"dt": 1e-5, "skin": 5e-4, "youngs": 5e6, "poisson": 0.45, "restitution": 0.3, "friction": 0.5}
    vol = np.array([4 / 3 * math.pi * r1 ** 3, 4 / 3 * math.pi * r2 ** 3])
    x = np.array([[0.0, 0.0, 0.0], [r1 + r2 - ov, 0.0, 0.0]])
    v = np.array([[0.05, 0.0, 0.0], [-0.02, 0.0, 0.0]])
    atoms = {"x": x, "v": v, "quat": np.array([[1.0, 0, 0, 0]] * 2), "angmom": np.zeros((2, 3)),
             "shape": np.array([[r1] * 3, [r2] * 3]), "blockiness": np.array([2.0, 2.0]),
             "rmass": vol * 2500.0, "inertia": np.array([[0.4 * m * r * r] * 3 for m, r in zip(vol * 2500, (r1, r2))]),
             "volume": vol}
    sc["atoms"] = atoms
    o = oracle.SqOracle(sc)
    o.setup()
    f = o.atoms()["f"]
    sp = S.sphere_pour(n=10)   # material tables of the sphere oracle: same E, nu, e, mu
    fi, ti, fj, tj, _ = oracle.pair_force(sp, x[0], x[1], v[0], v[1], np.zeros(3), np.zeros(3), r1, r2,
                                          atoms["rmass"][0], atoms["rmass"][1], shearupdate=0)
    assert np.allclose(f[0], fi, rtol=1e-9, atol=0) and np.allclose(f[1], fj, rtol=1e-9, atol=0)
    assert f[0][0] < 0.0   # i pushed away from j (+x neighbour)


def test_aligned_ellipsoids_overlap():
    """Two ellipsoids aligned on x touch at the ends of their x semi-axes."""
    pa = {"center": [0.0, 0.0, 0.0], "quat": [1.0, 0.0, 0.0, 0.0], "shape": [2e-3, 1e-3, 1e-3], "n": 2.0}
    pb = {"center": [3.49e-3, 0.0, 0.0], "quat": [1.0, 0.0, 0.0, 0.0], "shape": [1.5e-3, 1e-3, 1e-3], "n": 2.0}
    sol = oracle.sq_contact_point(pa, pb)
    assert sol["merit"] < 1e-10 and not sol["fail"]
    assert max(sol["fi"], sol["fj"]) < 0.0
    assert abs(sol["point"][1]) < 1e-12 and abs(sol["point"][2]) < 1e-12
    assert 1.99e-3 < sol["point"][0] < 2.0e-3


def test_shape_function_derivatives():
    rng = np.random.default_rng(0)
    q = S.random_quaternions(rng, 1)[0]
    p = {"center": [1e-4, -2e-4, 3e-4], "quat": q, "shape": [1.3e-3, 1.7e-3, 1.1e-3], "n": 5.3}
    x = np.array([8e-4, 6e-4, -5e-4])
    f, g, h = oracle.sq_shape_props(p, x)
    eps = 1e-9
    for k in range(3):
        d = np.zeros(3)
        d[k] = eps
        fp, gp, _ = oracle.sq_shape_props(p, x + d)
        fm, gm, _ = oracle.sq_shape_props(p, x - d)
        assert abs((fp - fm) / (2 * eps) - g[k]) <= 1e-5 * np.abs(g).max()
        assert np.max(np.abs((gp - gm) / (2 * eps) - h[:, k])) <= 1e-4 * np.abs(h).max()


def test_newton_solution_optimality():
    """Converged contact point: gradients antiparallel, equal shape
    functions, and the same point from homotopy and from a nearby guess."""
    rng = np.random.default_rng(4)
    qs = S.random_quaternions(rng, 20)
    for k in range(10):
        pa = {"center": [0.0, 0.0, 0.0], "quat": qs[2 * k], "shape": rng.uniform(1e-3, 2e-3, 3), "n": rng.uniform(2, 8)}
        d = rng.normal(size=3)
        d *= 3.0e-3 / np.linalg.norm(d)
        pb = {"center": d, "quat": qs[2 * k + 1], "shape": rng.uniform(1e-3, 2e-3, 3), "n": rng.uniform(2, 8)}
        sol = oracle.sq_contact_point(pa, pb)
        assert not sol["fail"] and sol["merit"] < 1e-10
        gi, gj = sol["gradi"], sol["gradj"]
        cos = gi @ gj / (np.linalg.norm(gi) * np.linalg.norm(gj))
        assert cos < -1 + 1e-9
        assert abs(sol["fi"] - sol["fj"]) <= 1e-5 * max(abs(sol["fi"]), abs(sol["fj"]))
        sol2 = oracle.sq_contact_point(pa, pb, guess=sol["point"] + 1e-6)
        assert np.max(np.abs(sol2["point"] - sol["point"])) < 1e-8


def test_asphere_free_rotation():
    """Torque-free rigid body: angular momentum is conserved exactly in
    direction and magnitude (to rounding) and the kinetic energy to O(dt^2)."""
    rng = np.random.default_rng(7)
    shape = np.array([[2e-3, 1.2e-3, 1e-3]])
    blk = np.array([3.5])
    vol = S.sq_volume(shape, blk)
    inert = S.sq_inertia(shape, blk, 2500.0)
    L0 = np.array([[3e-9, -2e-9, 4e-9]])
    sc = {"dt": 1e-5, "skin": 5e-4, "youngs": 5e6, "poisson": 0.45, "restitution": 0.3, "friction": 0.5,
          "atoms": {"x": np.zeros((1, 3)), "v": np.zeros((1, 3)), "quat": S.random_quaternions(rng, 1),
                    "angmom": L0, "shape": shape, "blockiness": blk, "rmass": vol * 2500.0, "inertia": inert,
                    "volume": vol}}
    o = oracle.SqOracle(sc)
    o.setup()
    a0 = o.atoms()
    e0 = 0.5 * a0["omega"][0] @ a0["angmom"][0]
    o.run(2000)
    a = o.atoms()
    assert np.max(np.abs(a["angmom"][0] - L0[0])) < 1e-20
    e = 0.5 * a["omega"][0] @ a["angmom"][0]
    assert abs(e - e0) < 1e-6 * e0
    assert abs(np.linalg.norm(a["quat"][0]) - 1.0) < 1e-14
