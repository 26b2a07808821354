"""Known-answer tests of the CPU oracle: analytic cases and symmetry laws
(the reference ships no tests, golden logs or fixtures).  They are a second
pin next to the digests of the reference's own state in
tests/golden/reference_digests.json."""
import math

import numpy as np
import pytest

import gb2_scenarios as S
import oracle


def base(n, box=(1.0, 1.0, 1.0), dt=1e-6, e=0.3, mu=0.5, E=5e6, nu=0.45, periodic=(0, 0, 0)):
    sc = {"dt": dt, "skin": 0.5e-3, "boxlo": [0.0, 0.0, 0.0], "boxhi": list(box), "periodic": list(periodic),
          "every": 1, "delay": 0, "check": 1, "sortfreq": 0, "sortbinsize": 0.0, "rolling_cdt": 0,
          "tangential_damping": 1, "fixes": []}
    sc.update(S._materials(1, E, nu, e, mu))
    return sc


def atoms(pos, vel, r=1e-3, rho=2500.0, omega=None):
    pos = np.asarray(pos, dtype=float)
    a = S._atoms(pos, np.full(len(pos), r), rho, np.asarray(vel, dtype=float), omega)
    return a


def test_hertz_static_overlap_on_plane():
    # m g = 4/3 Y* sqrt(R d) d  ->  d = (3 m g / (4 Y* sqrt(R)))^(2/3), wall: reff = R, Y* = E / (2 (1 - nu^2))
    r, rho, E, nu, g = 1e-3, 2500.0, 5e6, 0.45, 9.81
    sc = base(1, dt=2e-6, e=0.1)
    sc["atoms"] = atoms([[0.5, 0.5, r]], [[0.0, 0.0, 0.0]], r, rho)
    sc["fixes"] = [{"kind": "gravity", "magnitude": g, "vector": [0, 0, -1]},
                   {"kind": "wall_plane", "dim": 2, "pos": 0.0, "wall_type": 1}, {"kind": "nve_sphere"}]
    o = oracle.Oracle(sc)
    o.setup()
    o.run(60000)
    m = 4.0 / 3.0 * math.pi * r ** 3 * rho
    ystar = E / (2.0 * (1.0 - nu * nu))
    d_exact = (3.0 * m * g / (4.0 * ystar * math.sqrt(r))) ** (2.0 / 3.0)
    d = r - o.atoms()["x"][0, 2]
    assert abs(d - d_exact) / d_exact < 1e-6
    assert abs(o.atoms()["v"][0, 2]) < 1e-8


def test_head_on_restitution():
    # Hertz + velocity damping with beta from e: the rebound ratio is the requested e (to a few %)
    for e in (0.3, 0.7, 0.95):
        sc = base(2, dt=1e-7, e=e)
        v0 = 0.1
        sc["atoms"] = atoms([[0.5 - 1.0005e-3, 0.5, 0.5], [0.5 + 1.0005e-3, 0.5, 0.5]], [[v0, 0, 0], [-v0, 0, 0]])
        sc["fixes"] = [{"kind": "nve_sphere"}]
        o = oracle.Oracle(sc)
        o.setup()
        o.run(20000)
        v = o.atoms()["v"]
        ratio = (v[1, 0] - v[0, 0]) / (2 * v0)
        assert abs(ratio - e) < 0.05 * e + 0.02, (e, ratio)


def test_coulomb_cap_and_sign():
    # pressed sphere pair sliding: |Ft| <= mu |Fn|, and the friction opposes the slip
    sc = base(2, e=0.5, mu=0.3)
    xi, xj = [0.0, 0.0, 0.0], [1.99e-3, 0.0, 0.0]
    vi, vj = [0.0, 0.5, 0.0], [0.0, -0.5, 0.0]
    sh = np.zeros(3)
    for _ in range(200):
        fi, ti, fj, tj, sh = oracle.pair_force(sc, xi, xj, vi, vj, [0, 0, 0], [0, 0, 0], 1e-3, 1e-3, 1e-5, 1e-5,
                                               shear=sh)
    en = np.array([-1.0, 0.0, 0.0])
    fn = np.dot(fi, en)
    ft = fi - fn * en
    assert np.linalg.norm(ft) <= 0.3 * abs(fn) * (1 + 1e-12)
    assert abs(np.linalg.norm(ft) - 0.3 * abs(fn)) < 1e-9 * abs(fn)
    assert ft[1] < 0.0
    # Newton's third law for the force, torques from the two contact radii
    assert np.array_equal(fj, -fi)


def test_pair_swap_symmetry_bitwise():
    # evaluating a pair from the other side with negated shear is bit-identical
    rng = np.random.default_rng(4)
    sc = base(2)
    sc["rolling_cdt"] = 1
    sc["rollfriction"] = np.full((1, 1), 0.1)
    for _ in range(200):
        ri, rj = rng.uniform(0.5e-3, 2e-3, 2)
        xi = rng.normal(size=3) * 1e-3
        d = rng.normal(size=3)
        xj = xi + d / np.linalg.norm(d) * (ri + rj) * rng.uniform(0.95, 0.999)
        vi, vj, wi, wj = (rng.normal(size=3) * s for s in (0.1, 0.1, 50, 50))
        sh = rng.normal(size=3) * 1e-7
        fi, ti, fj, tj, shi = oracle.pair_force(sc, xi, xj, vi, vj, wi, wj, ri, rj, 1e-5, 2e-5, shear=sh.copy())
        gj, uj, gi, ui, shj = oracle.pair_force(sc, xj, xi, vj, vi, wj, wi, rj, ri, 2e-5, 1e-5, shear=-sh)
        assert np.array_equal(gj, fj) and np.array_equal(uj, tj)
        assert np.array_equal(shj, -shi)


def test_momentum_conserved_periodic():
    # no walls or gravity in a fully periodic box: total pair force vanishes
    sc = S.sphere_pour(n=448, seed=9, box=(0.02, 0.02, 0.02), spacing=(2.5e-3, 2.5e-3, 2.5e-3), vmax=0.5)
    sc["periodic"] = [1, 1, 1]
    sc["fixes"] = [{"kind": "nve_sphere"}]
    sc["atoms"]["x"][:, 2] = np.mod(sc["atoms"]["x"][:, 2], 0.02)
    o = oracle.Oracle(sc)
    o.setup()
    for _ in range(5):
        o.run(100)
        a = o.atoms()
        fs = np.abs(a["f"]).sum(axis=0)
        assert np.all(np.abs(a["f"].sum(axis=0)) <= 1e-12 * np.maximum(fs, 1e-30))
    p = o.pairs()
    assert (p["flag"] != 0).sum() > 0


def test_mesh_face_matches_plane():
    # a sphere resting on a flat two-triangle mesh floor settles at the plane's overlap
    r, rho = 1e-3, 2500.0
    sc = base(1, dt=2e-6, e=0.1)
    sc["atoms"] = atoms([[0.5, 0.5, r]], [[0.0, 0.0, 0.0]], r, rho)
    sq = [[[0.1, 0.1, 1e-9], [0.9, 0.1, 1e-9], [0.9, 0.9, 1e-9]], [[0.1, 0.1, 1e-9], [0.9, 0.9, 1e-9], [0.1, 0.9, 1e-9]]]
    sc["fixes"] = [{"kind": "gravity", "magnitude": 9.81, "vector": [0, 0, -1]},
                   {"kind": "wall_mesh", "nodes": np.array(sq), "wall_type": 1}, {"kind": "nve_sphere"}]
    o = oracle.Oracle(sc)
    o.setup()
    o.run(60000)
    sc2 = dict(sc)
    sc2["fixes"] = [sc["fixes"][0], {"kind": "wall_plane", "dim": 2, "pos": 1e-9, "wall_type": 1}, sc["fixes"][2]]
    o2 = oracle.Oracle(sc2)
    o2.setup()
    o2.run(60000)
    z1, z2 = o.atoms()["x"][0, 2], o2.atoms()["x"][0, 2]
    assert abs(z1 - z2) < 1e-12
    ea, ca, ob = o.mesh_topology(1, 2)
    assert ea.tolist() == [[1, 1, 0], [0, 1, 1]]   # shared coplanar diagonal inactive on both


def test_cone_topology_counts():
    sc = S.hopper(n=100, n_theta=64, n_z=16)
    o = oracle.Oracle(sc)
    ea, ca, ob = o.mesh_topology(1, len(sc["fixes"][1]["nodes"]))
    # ring edges between coplanar rows and quad diagonals are inactive; boundary rings active;
    # each generator line shared by two sectors is active on the larger element id only
    assert ea.sum() == 64 + 64 + 64 * 16
    assert ca.sum() == 2 * 64            # only boundary-ring nodes keep an active corner


def test_move_mesh_rotate_kinematics():
    """fix move/mesh rotate in the oracle: after k steps every node is the
    initial node turned by k*omega*dt about the axis (to rounding), and the
    node velocity is omega x r."""
    sc = S.drum(n=200, diameter=0.05, length=0.03, n_theta=24, n_ax=4, cap_rings=2, omega=30.0)
    n0 = np.asarray(sc["fixes"][1]["nodes"]).reshape(-1, 3, 3)
    o = oracle.Oracle(sc)
    o.setup()
    nodes, vel = o.mesh_nodes(1)
    assert np.array_equal(nodes, n0) and not vel.any()
    k = 400
    o.run(k)
    nodes, vel = o.mesh_nodes(1)
    phi = 30.0 * sc["dt"] * k
    c, s_ = np.cos(phi), np.sin(phi)
    rot = np.array([[1, 0, 0], [0, c, -s_], [0, s_, c]])
    expect = n0 @ rot.T
    assert np.max(np.abs(nodes - expect)) < 1e-12
    w = np.array([30.0, 0.0, 0.0])
    assert np.max(np.abs(vel - np.cross(w, nodes))) < 1e-13


def test_cylinder_wall_matches_plane():
    """A sphere pressed against a zcylinder wall from inside feels the same
    wall force as against a plane with the same overlap, pointing inward."""
    def one(fix):
        sc = S.sphere_pour(n=1)
        sc["periodic"] = [0, 0, 0]
        sc["boxlo"], sc["boxhi"] = [-0.05, -0.05, -0.05], [0.05, 0.05, 0.05]
        a = sc["atoms"]
        r, ov = 1e-3, 2e-5
        a["x"] = np.array([[0.02 - r + ov, 0.0, 0.0]])
        a["v"] = np.zeros((1, 3))
        sc["fixes"] = [fix, {"kind": "nve_sphere"}]
        o = oracle.Oracle(sc)
        o.setup()
        return o.atoms()["f"][0]
    fc = one({"kind": "wall_cylinder", "dim": 2, "radius": 0.02, "c1": 0.0, "c2": 0.0, "wall_type": 1})
    fp = one({"kind": "wall_plane", "dim": 0, "pos": 0.02, "wall_type": 1})
    assert fc[0] < 0 and abs(fc[1]) < 1e-15 and abs(fc[2]) < 1e-15
    assert abs(fc[0] - fp[0]) <= 1e-9 * abs(fp[0])


def test_pair_gran_local_keywords_periodic_pair():
    # two equal spheres touching through the periodic x boundary: one row
    # (kept from the side with the larger tag), pos remapped into the box,
    # contactPoint at the unremapped midpoint, contactArea = pi (r^2 - d^2/4),
    # delta = 2 r - d, a head-on force purely normal
    r = 1e-3
    sc = base(2, periodic=(1, 0, 0))
    sc["atoms"] = atoms([[0.0009, 0.5, 0.5], [0.9993, 0.5, 0.5]], [[-0.1, 0, 0], [0.1, 0, 0]], r=r)
    sc["fixes"] = [{"kind": "nve_sphere"}]
    o = oracle.Oracle(sc)
    o.setup()
    rows = o.pair_gran_local(0x1fff)
    assert rows.shape == (1, 41)
    row = rows[0]
    d = (1.0 - 0.9993) + 0.0009
    assert np.array_equal(row[0:3], [0.9993, 0.5, 0.5])
    assert row[3] == pytest.approx(0.0009, rel=1e-9) and np.array_equal(row[4:6], [0.5, 0.5])
    assert np.array_equal(row[6:12], [0.1, 0, 0, -0.1, 0, 0])
    assert np.array_equal(row[12:15], [2.0, 1.0, 1.0])
    F, fn, ft, T, tn, tt, h = (row[15:18], row[18:21], row[21:24], row[24:27], row[27:30], row[30:33], row[33:36])
    assert F[0] < 0 and F[1] == 0 and F[2] == 0
    assert fn == pytest.approx(F, rel=1e-14) and np.all(np.abs(ft) <= 1e-14 * abs(F[0]))
    assert np.array_equal(T, [0, 0, 0]) and np.array_equal(tn, [0, 0, 0]) and np.array_equal(tt, [0, 0, 0])
    assert np.array_equal(h, [0, 0, 0])
    assert row[36] == pytest.approx(math.pi * (r * r - d * d / 4), rel=1e-9)
    assert row[37] == pytest.approx(2 * r - d, rel=1e-9)
    assert row[38] == pytest.approx(1.0001, rel=1e-12) and np.array_equal(row[39:41], [0.5, 0.5])
    # the default id force torque history columns are the same numbers
    assert np.array_equal(o.pair_gran_local(), row[np.r_[12:18, 24:27, 33:36]][None, :])


def test_park_miller_minimal_standard():
    # Park & Miller (1988): from seed 1 the 10,000th state is 1043618065
    assert oracle.lib().orc_park_after(1, 10000) == 1043618065


@pytest.mark.parametrize("kw", [dict(), dict(periodic=False, vel_style="constant", all_in=1),
                                dict(target=("particles_in_region", 150), exact_number=0, vel_style="gaussian"),
                                dict(polydisperse=True, all_in=1), dict(cylinder=True, all_in=1)])
def test_insert_pack_places_non_overlapping_particles(kw):
    # fix insert/pack at the first step: the new particles lie in the region
    # (all_in: a radius away from its faces), overlap neither each other nor
    # the bed, follow the templates, and get tags after the bed's
    sc = S.insert_pour(**kw)
    n_bed = len(sc["atoms"]["tag"])
    fx = [f for f in sc["fixes"] if f["kind"] == "insert_pack"][0]
    o = oracle.Oracle(sc)
    o.setup()
    o.run(1)
    a = o.atoms()
    st = o.insert_stats()
    new = a["tag"] > n_bed
    k = int(new.sum())
    assert k == st["ninserted"] > 50 and st["next_step"] == 1 + fx["insert_every"]
    assert np.array_equal(np.sort(a["tag"][new]), np.arange(n_bed + 1, n_bed + k + 1))
    if "particles_in_region" in fx:
        # random_distribute uncorrelated draws each template's count
        slack = 0 if fx["exact_number"] else len(fx["templates"])
        assert abs(k - fx["particles_in_region"]) <= slack
    x = a["x"]
    # smallest radius a template can give (gaussian: cut at mean - 3 sigma)
    rad = np.array([t["radius"] - (3 * t["radius2"] if t.get("radius_style") == "gaussian" else 0.0)
                    for t in fx["templates"]])
    # radii from the masses (rmass = density * 4/3 pi r^3)
    xn = x[new]
    cyl = fx.get("region_cylinder")
    if cyl:
        rr = np.hypot(xn[:, 0] - cyl["c1"], xn[:, 1] - cyl["c2"])
        assert np.all(rr <= cyl["radius"]) and np.all((xn[:, 2] >= cyl["lo"]) & (xn[:, 2] <= cyl["hi"]))
        lo = np.array([cyl["c1"] - cyl["radius"], cyl["c2"] - cyl["radius"], cyl["lo"]])
        hi = np.array([cyl["c1"] + cyl["radius"], cyl["c2"] + cyl["radius"], cyl["hi"]])
    else:
        lo, hi = np.array(fx["region_lo"]), np.array(fx["region_hi"])
    assert np.all((xn >= lo) & (xn <= hi))
    vz = a["v"][new][:, 2]
    if kw.get("vel_style", "uniform") == "uniform":
        assert np.all(np.abs(a["v"][new] - [0, 0, -0.5]) <= 0.1 + 1e-9)
    elif kw.get("vel_style") == "constant":
        assert np.all(vz < 0)
    # gaps: new-new at least two of the smaller template radius, new-bed at
    # least that radius plus the bed's 1 mm (the bed has not moved since)
    d = np.linalg.norm(xn[:, None, :] - xn[None, :, :], axis=2)
    np.fill_diagonal(d, np.inf)
    assert d.min() > 2 * rad.min()
    db = np.linalg.norm(xn[:, None, :] - x[~new][None, :, :], axis=2)
    assert db.min() > rad.min() + 1e-3
    if fx.get("all_in"):
        gap = np.minimum(xn - lo, hi - xn).min(axis=1) if not cyl else np.minimum(
            cyl["radius"] - rr, np.minimum(xn[:, 2] - cyl["lo"], cyl["hi"] - xn[:, 2]))
        assert np.all(gap >= rad.min())
    r, m = o.radius_mass()
    rn, mn = r[new], m[new]
    assert np.allclose(mn, 2500.0 * 4.0 * np.pi / 3.0 * rn ** 3, rtol=1e-14)
    t0, t1 = fx["templates"]
    if kw.get("polydisperse"):
        # uniform template: radii in [1.0, 1.3] mm; gaussian: within 3 sigma of 0.8 mm
        big, small = rn[rn >= 0.95e-3], rn[rn < 0.95e-3]
        assert len(big) > 5 and len(small) > 20 and len(np.unique(rn)) > 0.9 * len(rn)
        assert big.min() >= t0["radius"] and big.max() <= t0["radius2"]
        assert np.all(np.abs(small - t1["radius"]) <= 3 * t1["radius2"] * (1 + 1e-12))
        assert abs(small.mean() - t1["radius"]) < 0.3 * t1["radius2"]
    else:
        assert set(np.unique(rn)) <= {t0["radius"], t1["radius"]}


def test_restart_carries_mesh_history():
    # write_restart / read_restart of the mesh contact history: a run
    # restarted from the restart layout (atoms, pair, plane-wall and mesh
    # histories) has, right after its setup, every mesh contact of the
    # original run with the same shear
    from parity_util import mesh_contact_map, restart_scenario
    sc = S.hopper(n=4000, n_theta=48, n_z=12, seed=5, gap=0.002, vmax=0.5)
    o = oracle.Oracle(sc)
    o.setup()
    o.run(900)
    before = mesh_contact_map(o.mesh_contacts(1))
    mh, he = o.mesh_history(1), o.history()
    assert mh["npartner"].sum() == len(before) > 20 and mh["npartner"].max() >= 2
    o2 = oracle.Oracle(restart_scenario(sc, o.atoms()))
    o2.upload_history(he["npartner"], he["partner_tag"], he["hist"])
    o2.upload_wall_hist(2, o.wall_hist(2))
    o2.upload_mesh_hist(1, mh["npartner"], mh["tri"], mh["hist"])
    o2.setup()
    assert mesh_contact_map(o2.mesh_contacts(1)) == before


def test_finnie_wear_linear_in_k():
    # wear finnie is non-negative, lands on the elements the particles touch,
    # and doubles bit for bit with k_finnie (only powers of two change)
    sc = S.silo(n=600, piston_speed=0.5)
    ntri = len(sc["fixes"][3]["nodes"])
    out = []
    for k in (0.5, 1.0):
        o = oracle.Oracle(sc)
        o.add_mesh_stress(3, [0.0, 0.0, 0.0])
        o.add_mesh_wear(3, np.full((sc["ntypes"], sc["ntypes"]), k))
        o.setup()
        o.run(1500)
        out.append(o.mesh_wear(3, ntri))
    assert np.all(out[0] >= 0) and out[0].max() > 0
    assert np.array_equal(out[1], 2 * out[0])
