"""Parity with the reference itself (LIGGGHTS-PUBLIC 3.8.0).

The reference is built from its own sources by oracle/Makefile.ref; the
harness (oracle/ref_harness.cpp) runs each scene's input script through the
reference library and dumps its raw state.  tests/golden/reference_digests.json
holds SHA-256 digests of those states (tests/golden/make_golden.py), so:

* CPU: the committed digests are what the reference produces today (when the
  reference is built here), and the oracle reproduces every checkpoint of
  every scene bit for bit: atoms (x, v, omega, f, torque in local order), the
  pair list with contact flags and shear history, primitive-wall histories,
  mesh contact slots, mesh nodes and node velocities, rebuild counts.
* GPU: the engine (FP64) reproduces the same digests, including the full
  config-1 pour (20,000 spheres, 20,000 steps); when the harness is present
  the engine is also compared state against state with a live reference run.

Bar: bit-identical for every compared quantity.
"""
import json
import os

import numpy as np
import pytest

import oracle
import ref
from ref_scenes import ALL_SCENES, RESTART_SCENES, SCENES, STREAM_SCENES, digest_dump, digest_sim, first_difference

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_digests.json")
with open(GOLDEN) as _f:
    DIGESTS = json.load(_f)


def _ref_available():
    try:
        return ref.build()
    except Exception:
        return False


def _run_checkpoints(sim, sc, segments, nbuilds, t0=0):
    out, t = [], t0
    sim.setup()
    for s in segments:
        if s:
            sim.run(s)
        t += s
        out.append(digest_sim(sc, sim, t, nbuilds(sim)))
    return out


def _compare(name, got):
    want = DIGESTS[name]["checkpoints"]
    assert len(got) == len(want)
    for k, (w, g) in enumerate(zip(want, got)):
        diff = first_difference(w, g)
        assert diff is None, "%s: checkpoint %d (step %d) differs from the reference: %s" % (
            name, k, w["ntimestep"], diff)


def test_golden_covers_every_scene():
    assert set(ALL_SCENES) <= set(DIGESTS)
    for name, (_, segments) in ALL_SCENES.items():
        assert DIGESTS[name]["segments"] == segments
    # the scenes exercise what they are for
    last = {k: DIGESTS[k]["checkpoints"][-1] for k in DIGESTS}
    assert last["hopper_mesh"]["nmesh1"] > 0 and last["drum_rotating"]["nmesh1"] > 0
    assert last["silo_cylinder_piston"]["nmesh3"] > 0
    assert last["insert_pack_periodic"]["nlocal"] > 400
    assert last["config1_pour_20k_20000steps"]["ntouch"] > 40000


def test_golden_covers_every_restart_scene():
    for name, (_, n_before, segments) in RESTART_SCENES.items():
        assert DIGESTS[name]["restart_after"] == n_before and DIGESTS[name]["segments"] == segments
        first = DIGESTS[name]["checkpoints"][0]
        assert first["ntimestep"] == n_before and first["ntouch"] > 0
    assert DIGESTS["drum_rotating_restart"]["checkpoints"][0]["nmesh1"] > 0
    assert DIGESTS["silo_cylinder_piston_restart"]["checkpoints"][0]["nmesh3"] > 0


@pytest.mark.parametrize("name", sorted(RESTART_SCENES))
def test_reference_restart_reproduces_golden(name):
    """The restart digests are the reference's output through a real
    restart file (write_restart, clear, read_restart; live run here)."""
    if not _ref_available():
        pytest.skip("reference not built and its sources are absent")
    build, n_before, segments = RESTART_SCENES[name]
    sc = build()
    _compare(name, [digest_dump(sc, d) for d in ref.run_restart(sc, n_before, segments)])


@pytest.mark.parametrize("name", sorted(SCENES) + sorted(STREAM_SCENES))
def test_reference_reproduces_golden(name):
    """The committed digests are the reference's output (live run here)."""
    if not _ref_available():
        pytest.skip("reference not built and its sources are absent")
    build, segments = ALL_SCENES[name]
    sc = build()
    got = [digest_dump(sc, d) for d in ref.run(sc, segments)]
    _compare(name, got)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_oracle_matches_reference(name):
    """The oracle equals the reference bit for bit at every checkpoint."""
    build, segments = SCENES[name]
    sc = build()
    o = oracle.Oracle(sc)
    _compare(name, _run_checkpoints(o, sc, segments, lambda s: s.nbuilds))


def test_oracle_matches_reference_state_by_state():
    """State-for-state comparison with a live reference run (readable
    failures): atoms, pairs, wall history and mesh slots on the hopper."""
    if not _ref_available():
        pytest.skip("reference not built and its sources are absent")
    build, segments = SCENES["hopper_mesh"]
    sc = build()
    dumps = ref.run(sc, segments[:3])
    o = oracle.Oracle(sc)
    o.setup()
    for s, d in zip(segments[:3], dumps):
        if s:
            o.run(s)
        a = o.atoms()
        assert np.array_equal(a["tag"], d["tag"])
        for k in ("x", "v", "omega", "f", "torque"):
            assert np.array_equal(a[k], d[k]), k
        p = o.pairs()
        assert np.array_equal(p["tag_j"], d["pair_j"]) and np.array_equal(p["hist"], d["pair_hist"])
        mc = o.mesh_contacts(1)
        assert np.array_equal(mc["tri"], d["w0_tri"]) and np.array_equal(mc["hist"], d["w0_hist"])
        assert np.array_equal(o.mesh_geom(1), d["w0_geom"]), "element geometry differs"
        assert np.array_equal(o.wall_hist(2), d["w1_hist"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(ALL_SCENES))
def test_engine_matches_reference(name):
    """The engine (FP64) equals the reference bit for bit at every checkpoint."""
    import granb200
    build, segments = ALL_SCENES[name]
    sc = build()
    e = granb200.Engine(sc)
    _compare(name, _run_checkpoints(e, sc, segments, lambda s: s.stats()["nbuilds"]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["hopper_packed_discharge", "bidisperse_long_lists", "insert_pack_periodic"])
def test_engine_mask_rounds_match_reference(name, monkeypatch):
    """The pair step's other enumeration: with the per-warp item lists
    disabled (GB2_ITEM_CAP=0, as a warp whose lists outgrow their capacity
    runs) every warp evaluates its pairs from the screening bitmasks; the
    results are the same digests, bit for bit."""
    import granb200
    monkeypatch.setenv("GB2_ITEM_CAP", "0")
    build, segments = ALL_SCENES[name]
    sc = build()
    e = granb200.Engine(sc)
    _compare(name, _run_checkpoints(e, sc, segments, lambda s: s.stats()["nbuilds"]))
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(RESTART_SCENES))
def test_engine_restart_matches_reference(name):
    """A restart: the engine runs n_before steps, its state is downloaded
    in the restart layout (atoms in local order, pair contact history as
    partner tags and shear, primitive-wall histories, mesh contact slots,
    current mesh nodes), and a new engine built from that download equals,
    bit for bit at every checkpoint, the reference continued from its own
    restart file (the restarted setup re-sorts the atoms and computes forces
    without a shear update, as every setup does, and the atom-sort schedule
    counts from the restart's timestep)."""
    import granb200
    build, n_before, segments = RESTART_SCENES[name]
    sc = build()
    e = granb200.Engine(sc)
    e.setup()
    e.run(n_before)
    snap = e.snapshot(sc)
    e.close()
    assert snap["ntimestep"] == n_before
    sc2 = granb200.restart_scenario(sc, snap["atoms"], {i: m["nodes"] for i, m in snap["meshes"].items()},
                                    ntimestep=snap["ntimestep"])
    e2 = granb200.Engine(sc2)
    e2.restore(snap)
    _compare(name, _run_checkpoints(e2, sc2, segments, lambda s: s.stats()["nbuilds"], t0=n_before))


@pytest.mark.gpu
def test_engine_matches_live_reference_drum():
    """State against state with a live reference run, when the harness is on
    this machine: the rotating drum (moving-mesh geometry refreshed at every
    rebuild, barycentric wall velocities, mesh slots)."""
    if not ref.available():
        pytest.skip("reference harness not present on this machine")
    import granb200
    build, segments = SCENES["drum_rotating"]
    sc = build()
    dumps = ref.run(sc, segments)
    e = granb200.Engine(sc)
    e.setup()
    for s, d in zip(segments, dumps):
        if s:
            e.run(s)
        a = e.atoms()
        assert np.array_equal(a["tag"], d["tag"])
        for k in ("x", "v", "omega", "f", "torque"):
            assert np.array_equal(a[k], d[k]), "%s differs at step %d" % (k, d["ntimestep"])
        mc = e.mesh_contacts(1)
        assert np.array_equal(mc["tri"], d["w0_tri"]) and np.array_equal(mc["hist"], d["w0_hist"])
