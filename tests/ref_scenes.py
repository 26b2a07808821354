"""Scenes run through the reference itself, and how their states are compared.

Each scene is a seeded scenario (the package's scenario generators) plus a
list of run segments: setup (segment 0, zero steps) and the further runs
after which the state is checked.  ``digest`` reduces one checkpoint of any
run (reference harness dump, oracle or engine download) to SHA-256 digests of
its raw bytes, so a committed fixture pins bit-exact equality without
shipping the state itself.
"""
import hashlib

import numpy as np

import gb2_scenarios as S


def _pour3k():
    sc = S.sphere_pour(n=3000, seed=11, omega_max=20.0)
    sc["sortfreq"] = 100
    sc["rolling_cdt"] = 1
    sc["fixes"][1]["rolling_cdt"] = 1
    sc["rollfriction"] = np.full((1, 1), 0.1)
    return sc


def _two_types():
    sc = S.sphere_pour(n=2000, seed=21, vmax=0.3)
    n = len(sc["atoms"]["tag"])
    sc["atoms"]["type"] = np.where(np.arange(n) % 3 == 0, 2, 1).astype(np.int32)
    sc["ntypes"] = 2
    sc["youngs"] = np.array([5e6, 2e7])
    sc["poisson"] = np.array([0.45, 0.3])
    sc["restitution"] = np.array([[0.3, 0.5], [0.5, 0.7]])
    sc["friction"] = np.array([[0.5, 0.2], [0.2, 0.4]])
    sc["rollfriction"] = np.zeros((2, 2))
    sc["every"], sc["delay"], sc["check"] = 3, 6, 1
    sc["tangential_damping"] = 0
    return sc


def _hopper_mesh():
    sc = S.hopper(n=4000, n_theta=48, n_z=12, seed=5, gap=0.002, vmax=0.5)
    sc["sortfreq"] = 200
    return sc


def _drum():
    sc = S.drum(n=1500, diameter=0.05, length=0.03, n_theta=48, n_ax=12, cap_rings=3, omega=50.0,
                clearance=0.3e-3, vmax=0.05)
    sc["sortfreq"] = 300
    return sc


def _hopper_packed():
    return S.hopper_packed(n=6000, n_theta=48, n_z=12, band=0.02, sortfreq=200)


def _drum_config3():
    return S.drum_config3(n=6000, diameter=0.06, length=0.05, n_theta=48, n_ax=12, cap_rings=3, band=0.02,
                          omega=20.0, sortfreq=300)


def _bed_config5():
    return S.bed_config5(n=20000, box=(0.02, 0.02, 0.05), plate_nx=32, plate_ny=32, plate_waves=(2, 2),
                         sortfreq=300)


# name -> (scenario builder, run segments); segment 0 is the setup
SCENES = {
    "hopper_packed_discharge": (_hopper_packed, [0, 200, 200, 200, 200, 200]),
    "drum_config3_packed": (_drum_config3, [0, 300, 300, 300, 300]),
    "bed_config5_packed": (_bed_config5, [0, 300, 300, 300]),
    "pour3k_rolling": (_pour3k, [0, 150, 150, 150, 150]),
    "two_types_schedule": (_two_types, [0, 300, 300, 300, 300]),
    "hopper_mesh": (_hopper_mesh, [0, 300, 300, 300, 300, 300]),
    "drum_rotating": (_drum, [0, 500, 500, 500, 500, 500, 500, 500, 500]),
    "silo_cylinder_piston": (lambda: S.silo(n=1500, piston_speed=0.5), [0, 500, 500, 500, 500, 500, 500]),
    "bidisperse_long_lists": (S.bidisperse_bed, [0, 250, 250, 250, 250, 250, 250]),
    "insert_pack_periodic": (lambda: S.insert_pour(insert_every=250), [0, 300, 300, 300, 300]),
    "insert_pack_walled_all_in": (lambda: S.insert_pour(periodic=False, vel_style="constant", all_in=1),
                                  [0, 300, 300, 300, 300]),
    "insert_pack_count_gaussian": (lambda: S.insert_pour(target=("particles_in_region", 150), exact_number=0,
                                                         vel_style="gaussian", insert_every=200),
                                   [0, 300, 300, 300, 300]),
    "insert_pack_cylinder_mass": (lambda: S.insert_pour(cylinder=True, target=("mass_in_region", 0.003),
                                                        insert_every=250), [0, 300, 300, 300, 300]),
}

# fix insert/stream: the reference (live, CPU) and the engine (GPU) are
# compared with the digests; the oracle restates insert/pack only
STREAM_SCENES = {
    "stream_insert_periodic": (S.stream_pour, [0, 300, 300, 300, 300, 300]),
    "stream_insert_walled": (lambda: S.stream_pour(periodic=False, vel_style="constant", exact_number=0,
                                                   particlerate=15000.0, vel=(0.0, 0.0, -1.5)),
                             [0, 300, 300, 300, 300, 300]),
}

# Too long for the reference or the oracle inside the CPU test run (the
# reference needs ~110 s); pinned by committed digests and run on the GPU.
LONG_SCENES = {
    "config1_pour_20k_20000steps": (S.sphere_pour, [0, 20000]),
    "config2_hopper_1M_100steps": (S.hopper_packed, [0, 100]),
}

ALL_SCENES = dict(SCENES, **STREAM_SCENES, **LONG_SCENES)

# Restart through a real restart file: the reference runs n_before steps,
# write_restart, clear, read_restart, then the segments (setup first); the
# engine restarts from its own download of the same state (atoms, pair,
# primitive-wall and mesh contact histories, current mesh nodes).
# name -> (scenario builder, n_before, segments after the restart)
RESTART_SCENES = {
    "drum_rotating_restart": (_drum, 2500, [0, 500, 500]),
    "silo_cylinder_piston_restart": (lambda: S.silo(n=1500, piston_speed=0.5), 1500, [0, 500, 500]),
    "pour3k_rolling_restart": (_pour3k, 300, [0, 150, 150]),
}


def _h(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def walls(sc):
    """Scenario fix indices of the wall/gran fixes, in definition order."""
    return [i for i, f in enumerate(sc["fixes"]) if f["kind"] in ("wall_plane", "wall_cylinder", "wall_mesh")]


def digest_dump(sc, d):
    """Digests of one reference harness dump."""
    out = {"ntimestep": int(d["ntimestep"]), "nbuilds": int(d["ncalls"]) + 1, "nlocal": int(d["nlocal"]),
           "npairs": int(len(d["pair_i"])), "ntouch": int((d["pair_flag"] != 0).sum()),
           "atoms": _h(d["tag"].astype(np.int32), d["x"], d["v"], d["omega"], d["f"], d["torque"]),
           "pairs": _h(d["pair_i"].astype(np.int32), d["pair_j"].astype(np.int32),
                       d["pair_flag"].astype(np.int32), d["pair_hist"].reshape(-1, 3))}
    for k, ifix in enumerate(walls(sc)):
        if sc["fixes"][ifix]["kind"] == "wall_mesh":
            out["wall%d" % ifix] = _h(d["w%d_tag" % k].astype(np.int32), d["w%d_tri" % k].astype(np.int32),
                                      d["w%d_hist" % k].reshape(-1, 3))
            out["nodes%d" % ifix] = _h(d["w%d_nodes" % k].reshape(-1, 3, 3), d["w%d_vnode" % k].reshape(-1, 3, 3))
            out["nmesh%d" % ifix] = int(len(d["w%d_tag" % k]))
        else:
            out["wall%d" % ifix] = _h(d["w%d_hist" % k].reshape(-1, 3))
    return out


def digest_sim(sc, sim, ntimestep, nbuilds):
    """The same digests of an oracle or engine state (same accessor names)."""
    a = sim.atoms()
    p = sim.pairs()
    out = {"ntimestep": int(ntimestep), "nbuilds": int(nbuilds), "nlocal": int(len(a["tag"])),
           "npairs": int(len(p["tag_i"])), "ntouch": int((p["flag"] != 0).sum()),
           "atoms": _h(a["tag"].astype(np.int32), a["x"], a["v"], a["omega"], a["f"], a["torque"]),
           "pairs": _h(p["tag_i"].astype(np.int32), p["tag_j"].astype(np.int32), p["flag"].astype(np.int32),
                       np.asarray(p["hist"]).reshape(-1, 3))}
    for ifix in walls(sc):
        if sc["fixes"][ifix]["kind"] == "wall_mesh":
            mc = sim.mesh_contacts(ifix)
            out["wall%d" % ifix] = _h(mc["tag"].astype(np.int32), mc["tri"].astype(np.int32),
                                      np.asarray(mc["hist"]).reshape(-1, 3))
            nodes, vel = sim.mesh_nodes(ifix)
            out["nodes%d" % ifix] = _h(np.asarray(nodes).reshape(-1, 3, 3), np.asarray(vel).reshape(-1, 3, 3))
            out["nmesh%d" % ifix] = int(len(mc["tag"]))
        else:
            out["wall%d" % ifix] = _h(np.asarray(sim.wall_hist(ifix)).reshape(-1, 3))
    return out


def first_difference(want, got):
    """Name of the first differing digest entry (None when equal)."""
    for k in want:
        if want[k] != got.get(k):
            return "%s (%r vs %r)" % (k, want[k], got.get(k))
    return None
