"""Engine (CUDA, FP64) vs oracle parity on small seeded workloads.

FP64 bar: bit-identical.  The engine evaluates the reference arithmetic in
the reference order with FMA contraction off, so positions, velocities,
forces, torques, neighbour pairs, contact flags and every shear-history slot
must equal the oracle bit for bit, including across neighbour rebuilds,
atom sorts and periodic images.
"""
import numpy as np
import pytest

import gb2_scenarios as S
import oracle
from parity_util import assert_atoms_equal, assert_mesh_equal, assert_pairs_equal

pytestmark = pytest.mark.gpu


def _pair(sc):
    import granb200
    e = granb200.Engine(sc)
    o = oracle.Oracle(sc)
    return e, o


def test_sphere_pour_setup():
    sc = S.sphere_pour(n=3000, seed=7)
    e, o = _pair(sc)
    e.setup()
    o.setup()
    assert_atoms_equal(e, o)
    assert_pairs_equal(e, o)


@pytest.mark.parametrize("rolling", [0, 1])
def test_sphere_pour_run(rolling):
    sc = S.sphere_pour(n=3000, seed=11, omega_max=20.0)
    sc["sortfreq"] = 100
    sc["rolling_cdt"] = rolling
    sc["fixes"][1]["rolling_cdt"] = rolling
    sc["rollfriction"] = np.full((1, 1), 0.1)
    e, o = _pair(sc)
    e.setup()
    o.setup()
    for _ in range(4):
        e.run(150)
        o.run(150)
        assert_atoms_equal(e, o)
        npairs, ntouch = assert_pairs_equal(e, o)
        assert np.array_equal(e.wall_hist(1), o.wall_hist(1))
    assert ntouch > 0 and o.nbuilds > 2
    assert e.stats()["nbuilds"] == o.nbuilds


def test_hopper_mesh_run():
    sc = S.hopper(n=4000, n_theta=48, n_z=12, seed=5)
    sc["sortfreq"] = 200
    e, o = _pair(sc)
    ea, ca, ob = e.mesh_topology(1)
    eo, co, oo = o.mesh_topology(1, len(sc["fixes"][1]["nodes"]))
    assert np.array_equal(ea, eo) and np.array_equal(ca, co) and np.array_equal(ob, oo)
    e.setup()
    o.setup()
    total = 0
    for _ in range(5):
        e.run(200)
        o.run(200)
        assert_atoms_equal(e, o)
        assert_pairs_equal(e, o)
        total += assert_mesh_equal(e, o, 1)
        assert np.array_equal(e.wall_hist(2), o.wall_hist(2))
    assert total > 0


def test_drum_rotating_mesh():
    """fix move/mesh rotate: mesh nodes and node velocities, the forced
    rebuilds when the mesh has moved more than skin/2, the moving-wall
    velocity at each contact and the mesh contact history, bit for bit."""
    sc = S.drum(n=1500, diameter=0.05, length=0.03, n_theta=48, n_ax=12, cap_rings=3, omega=50.0,
                clearance=0.3e-3, vmax=0.05)
    sc["sortfreq"] = 300
    e, o = _pair(sc)
    e.setup()
    o.setup()
    total = 0
    for _ in range(8):
        e.run(500)
        o.run(500)
        assert_atoms_equal(e, o)
        assert_pairs_equal(e, o)
        total += assert_mesh_equal(e, o, 1)
        en, ev = e.mesh_nodes(1)
        on, ov = o.mesh_nodes(1)
        assert np.array_equal(en, on) and np.array_equal(ev, ov), "mesh nodes or node velocities differ"
    assert total > 0, "no particle reached the rotating wall"
    assert e.stats()["nbuilds"] == o.nbuilds and o.nbuilds > 50


def test_deterministic():
    sc = S.sphere_pour(n=2000, seed=3)
    a = __import__("granb200").Engine(sc)
    b = __import__("granb200").Engine(sc)
    for x in (a, b):
        x.setup()
        x.run(300)
    pa, pb = a.atoms(), b.atoms()
    for k in ("x", "v", "omega", "f", "torque"):
        assert np.array_equal(pa[k], pb[k])


def test_silo_cylinder_wall_and_linear_piston():
    """zcylinder primitive wall (inside contact), floor plane and a
    triangulated piston driven by fix move/mesh linear, bit for bit."""
    sc = S.silo(n=1500, piston_speed=0.5)
    e, o = _pair(sc)
    e.setup()
    o.setup()
    for _ in range(6):
        e.run(500)
        o.run(500)
        assert_atoms_equal(e, o)
        assert_pairs_equal(e, o)
        assert np.array_equal(e.wall_hist(1), o.wall_hist(1)), "cylinder wall history differs"
        assert np.array_equal(e.wall_hist(2), o.wall_hist(2))
        assert_mesh_equal(e, o, 3)
        en, ev = e.mesh_nodes(3)
        on, ov = o.mesh_nodes(3)
        assert np.array_equal(en, on) and np.array_equal(ev, ov)
    assert np.abs(o.wall_hist(1)).sum() > 0, "no particle touched the cylinder"
    assert len(o.mesh_contacts(3)["tag"]) > 0, "the piston touched nothing"
    assert e.stats()["nbuilds"] == o.nbuilds


def test_bidisperse_long_lists_serial_path():
    """Two 3 mm spheres buried in a bed of 0.3 mm ones: each has ~177
    neighbour-list pairs, more than 64 on a side, so its pairs are evaluated
    serially in the reference order by the tail kernel; bit for bit."""
    import granb200
    sc = S.bidisperse_bed()
    e, o = _pair(sc)
    e.setup()
    o.setup()
    p = o.pairs()
    tags, counts = np.unique(np.concatenate([p["tag_i"], p["tag_j"]]), return_counts=True)
    assert counts.max() > 128, "no atom with a long list"
    big_touch = pgl_rows = pgl_periodic = 0
    for _ in range(6):
        e.run(250)
        o.run(250)
        assert_atoms_equal(e, o)
        assert_pairs_equal(e, o)
        q = o.pairs()
        big = np.isin(q["tag_i"], [1, 2]) | np.isin(q["tag_j"], [1, 2])
        big_touch += int(((q["flag"] != 0) & big).sum())
        assert np.array_equal(e.wall_hist(1), o.wall_hist(1))
        ca, cb = e.contact_atom(), o.contact_atom()
        assert np.array_equal(ca["tag"], cb["tag"]) and np.array_equal(ca["contact"], cb["contact"])
        ra, rb = e.pair_gran_local(), o.pair_gran_local()
        assert ra.shape == rb.shape and np.array_equal(ra, rb), "pair/gran/local rows differ"
        pgl_rows += len(rb)
        pgl_periodic += int(rb[:, 2].sum())
        # every keyword at once (pos remapped into the periodic box, the
        # normal / tangential splits, contactArea, delta, contactPoint)
        names = [k for k, _ in granb200.PGL_KEYWORDS]
        ka, kb = e.pair_gran_local(names), o.pair_gran_local(granb200.pgl_keys(names))
        assert ka.shape == kb.shape == (len(rb), 41) and np.array_equal(ka, kb), "pair/gran/local keyword rows differ"
        cols = granb200.pgl_columns(granb200.pgl_keys(names))
        assert np.array_equal(ka[:, cols.index("id[0]"):cols.index("id[0]") + 3], ra[:, :3])
        pos = ka[:, :6].reshape(-1, 2, 3)
        lo, hi = np.asarray(sc["boxlo"]), np.asarray(sc["boxhi"])
        per = np.asarray(sc["periodic"], dtype=bool)
        assert np.all((pos[..., per] >= lo[per]) & (pos[..., per] < hi[per])), "pos not remapped into the box"
        fn = ka[:, cols.index("force_normal[0]"):][:, :3]
        ft = ka[:, cols.index("force_tangential[0]"):][:, :3]
        assert np.allclose(fn + ft, ra[:, 3:6], rtol=1e-12, atol=1e-18)
        dl = ka[:, cols.index("delta")]
        assert np.all(dl > 0) and np.all(np.isfinite(ka[:, cols.index("contactArea")]))
    assert big_touch > 0, "the large spheres touched nothing"
    assert e.contact_atom()["contact"].max() > 10, "no large sphere with many contacts"
    assert pgl_rows > 100 and pgl_periodic > 0, "pair/gran/local saw too few pairs"
    assert e.stats()["nbuilds"] == o.nbuilds


def test_two_types_neighbor_schedule_no_tangential_damping():
    """Two atom types with different materials (type-pair lookups in both
    orders), neigh_modify every 3 delay 6 check yes and every 5 check no
    (the decide() schedule without the queue), tangential damping off;
    bit for bit, including the rebuild count."""
    for every, delay, check in ((3, 6, 1), (5, 0, 0)):
        sc = S.sphere_pour(n=2000, seed=21, vmax=0.3)
        n = len(sc["atoms"]["tag"])
        sc["atoms"]["type"] = np.where(np.arange(n) % 3 == 0, 2, 1).astype(np.int32)
        sc["ntypes"] = 2
        sc["youngs"] = np.array([5e6, 2e7])
        sc["poisson"] = np.array([0.45, 0.3])
        sc["restitution"] = np.array([[0.3, 0.5], [0.5, 0.7]])
        sc["friction"] = np.array([[0.5, 0.2], [0.2, 0.4]])
        sc["rollfriction"] = np.array([[0.0, 0.0], [0.0, 0.0]])
        sc["every"], sc["delay"], sc["check"] = every, delay, check
        sc["tangential_damping"] = 0
        e, o = _pair(sc)
        e.setup()
        o.setup()
        for _ in range(4):
            e.run(300)
            o.run(300)
            assert_atoms_equal(e, o)
            assert_pairs_equal(e, o)
        assert e.stats()["nbuilds"] == o.nbuilds > 1


def _restart_scenario(sc, atoms):
    from parity_util import restart_scenario
    return restart_scenario(sc, atoms)


def test_restart_history_roundtrip():
    """Restart interoperability: the contact history downloaded in
    FixContactHistory's partner layout equals the oracle's, and a run
    restarted from it (atoms, partner history, wall history) matches the
    oracle restarted from the same data bit for bit; right after the restart
    every touching pair carries the shear it had before."""
    sc = S.sphere_pour(n=2000, seed=8, vmax=0.3)
    e, o = _pair(sc)
    e.setup()
    o.setup()
    e.run(700)
    o.run(700)
    assert_atoms_equal(e, o)
    he, ho = e.history(), o.history()
    for k in ("tag", "npartner", "partner_tag", "hist"):
        assert np.array_equal(he[k], ho[k]), "history %s differs from the oracle" % k
    assert he["npartner"].sum() > 100, "too few contacts to test a restart"
    before = e.pairs()
    sc2 = _restart_scenario(sc, e.atoms())
    wall = e.wall_hist(1)
    import granb200
    e2, o2 = granb200.Engine(sc2), oracle.Oracle(sc2)
    for x in (e2, o2):
        x.upload_history(he["npartner"], he["partner_tag"], he["hist"])
        x.upload_wall_hist(1, wall)
        x.setup()
    assert_atoms_equal(e2, o2)
    assert_pairs_equal(e2, o2)
    after = e2.pairs()
    key = {(i, j): h for i, j, h, f in zip(before["tag_i"], before["tag_j"], before["hist"], before["flag"]) if f}
    carried = 0
    for i, j, h, f in zip(after["tag_i"], after["tag_j"], after["hist"], after["flag"]):
        if f and (i, j) in key:
            assert np.array_equal(h, key[(i, j)]), "shear of pair %d-%d not carried over" % (i, j)
            carried += 1
        elif f and (j, i) in key:
            assert np.array_equal(h, -key[(j, i)]), "shear of pair %d-%d not carried over" % (i, j)
            carried += 1
    assert carried > 50
    for _ in range(3):
        e2.run(300)
        o2.run(300)
        assert_atoms_equal(e2, o2)
        assert_pairs_equal(e2, o2)


def test_mesh_surface_stress():
    """fix mesh/surface/stress on the silo piston: per-triangle force and the
    mesh's total force and torque about a reference point, each step; the
    device sums in another order (atomics), so they equal the oracle to
    1e-12 of the largest value, not bit for bit."""
    sc = S.silo(n=1500, piston_speed=0.5)
    e, o = _pair(sc)
    kf = np.full((sc["ntypes"], sc["ntypes"]), 0.7)
    for x in (e, o):
        x.add_mesh_stress(3, [0.001, -0.002, 0.01])
        x.add_mesh_wear(3, kf)
        x.setup()
    ntri = len(sc["fixes"][3]["nodes"])
    hits = 0
    for _ in range(6):
        e.run(500)
        o.run(500)
        assert_atoms_equal(e, o)
        a, b = e.mesh_stress(3), o.mesh_stress(3)
        scale = max(np.abs(b["tri_f"]).max(), 1e-30)
        assert np.abs(a["tri_f"] - b["tri_f"]).max() <= 1e-12 * scale
        assert np.abs(a["f_total"] - b["f_total"]).max() <= 1e-12 * max(np.abs(b["f_total"]).max(), scale)
        tq = max(np.abs(b["torque_total"]).max(), 1e-30)
        assert np.abs(a["torque_total"] - b["torque_total"]).max() <= 1e-12 * tq
        for k in ("sigma_n", "sigma_t"):
            assert np.abs(a[k] - b[k]).max() <= 1e-10 * max(np.abs(b[k]).max(), 1e-30), k
        hits += int((np.abs(b["tri_f"]).sum(axis=1) > 0).sum())
        # Finnie wear, cumulative per element (atomics: to 1e-12 of the largest)
        wa, wb = e.mesh_wear(3), o.mesh_wear(3, ntri)
        assert np.abs(wa - wb).max() <= 1e-12 * max(wb.max(), 1e-300)
    assert hits > 0, "the piston carried no force"
    assert wb.max() > 0 and np.all(wb >= 0), "no wear on the piston"
    assert b["f_total"][2] > 0, "particles should push the piston up"
    # restart of the wear: two restarts of the same snapshot, one with the
    # cumulative wear uploaded; after setup they differ by exactly that wear
    import granb200
    snap = e.snapshot(sc)
    sc2 = granb200.restart_scenario(sc, snap["atoms"], {i: m["nodes"] for i, m in snap["meshes"].items()})
    w = []
    for up in (True, False):
        x = granb200.Engine(sc2)
        x.restore(snap)
        x.add_mesh_stress(3, [0.001, -0.002, 0.01])
        x.add_mesh_wear(3, kf)
        if up:
            x.upload_mesh_wear(3, wa)
        x.setup()
        w.append(x.mesh_wear(3))
        x.close()
    assert np.abs((w[0] - w[1]) - wa).max() <= 1e-12 * wa.max()


def test_upload_rejects_bad_atoms():
    """An atom type outside 1..ntypes, a zero radius or a non-finite
    position is refused by the upload with its reason (the checks run while
    the copies are in flight), and a context whose upload failed has no atoms."""
    import granb200
    cases = [("type", 0, "atom type out of range"), ("radius", 0.0, "extended particles"),
             ("x", np.nan, "non-finite atom state")]
    for key, value, msg in cases:
        sc = S.sphere_pour(n=200, seed=3)
        a = dict(sc["atoms"])
        arr = np.array(a[key], copy=True)
        arr[7] = value
        a[key] = arr
        sc["atoms"] = a
        with pytest.raises(granb200.GB2Error, match=msg):
            granb200.Engine(sc)


def test_mesh_wear_needs_a_type_matrix():
    """k_finnie is an ntypes x ntypes matrix; anything else is refused before it reaches the library."""
    import granb200
    sc = S.silo(n=200, piston_speed=0.5)
    e = granb200.Engine(sc)
    e.add_mesh_stress(3, [0.0, 0.0, 0.0])
    with pytest.raises(ValueError):
        e.add_mesh_wear(3, np.full(sc["ntypes"] * sc["ntypes"] - 1, 0.7))
    e.close()


@pytest.mark.parametrize("kw", [dict(insert_every=250),
                                dict(periodic=False, vel_style="constant", all_in=1),
                                dict(target=("particles_in_region", 150), exact_number=0, vel_style="gaussian",
                                     insert_every=200),
                                dict(polydisperse=True, all_in=1, insert_every=250),
                                dict(cylinder=True, target=("mass_in_region", 0.003), insert_every=250)])
def test_insert_pack(kw):
    """fix insert/pack refilling a region block above a bed (periodic x/y with
    ghosts near the region, or walled; vel uniform / constant / gaussian;
    volume-fraction or count target; insertion steps at run starts and in
    the middle of a run): the same particles appear at the same steps with
    the same tags, and every state stays bit for bit equal to the oracle."""
    sc = S.insert_pour(**kw)
    e, o = _pair(sc)
    e.setup()
    o.setup()
    n0 = len(sc["atoms"]["tag"])
    for _ in range(4):
        e.run(300)
        o.run(300)
        assert e.insert_stats() == o.insert_stats()
        assert_atoms_equal(e, o)
        assert_pairs_equal(e, o)
    assert o.insert_stats()["ninserted"] > 100 and o.nlocal > n0
    assert e.stats()["nbuilds"] == o.nbuilds


def test_restart_mesh_history_roundtrip():
    """Restart of the mesh contact history: the restart layout (slots sorted
    as write_restart does) equals the oracle's, and a run restarted from it
    with the pair and wall histories matches the oracle restarted from the
    same data bit for bit, every mesh contact carried over with its shear."""
    from parity_util import mesh_contact_map, restart_scenario
    sc = S.hopper(n=4000, n_theta=48, n_z=12, seed=5, gap=0.002, vmax=0.5)
    e, o = _pair(sc)
    e.setup()
    o.setup()
    e.run(900)
    o.run(900)
    me, mo = e.mesh_history(1), o.mesh_history(1)
    for k in ("tag", "npartner", "tri", "hist"):
        assert np.array_equal(me[k], mo[k]), "mesh history %s differs from the oracle" % k
    assert me["npartner"].sum() > 20
    assert_mesh_equal(e, o, 1)
    before = mesh_contact_map(e.mesh_contacts(1))
    he = e.history()
    import granb200
    sc2 = restart_scenario(sc, e.atoms())
    e2, o2 = granb200.Engine(sc2), oracle.Oracle(sc2)
    for x in (e2, o2):
        x.upload_history(he["npartner"], he["partner_tag"], he["hist"])
        x.upload_wall_hist(2, e.wall_hist(2))
        x.upload_mesh_hist(1, me["npartner"], me["tri"], me["hist"])
        x.setup()
    assert mesh_contact_map(e2.mesh_contacts(1)) == before
    assert_atoms_equal(e2, o2)
    for _ in range(3):
        e2.run(300)
        o2.run(300)
        assert_atoms_equal(e2, o2)
        assert_pairs_equal(e2, o2)
        assert_mesh_equal(e2, o2, 1)
