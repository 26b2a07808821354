"""The drop-in boundary: the b200 suffix styles compiled into the reference.

liggghts-public_b200/lammps holds pair gran/b200, fix wall/gran/b200,
mesh/surface/b200, gravity/b200, move/mesh/b200, nve/sphere/b200 and run_style
verlet/b200.  oracle/Makefile.ref (target b200) drops them into a build of the
reference (style headers regenerated, factories recompiled) linked with
libgranb200.so, the way a maintainer adds them to src/.

CPU: "-sf b200" selects the styles through the reference's own factories
(Force::new_pair, Modify::add_fix, Update::create_integrate) and keywords
outside the accelerated path stop the run with error->all; without the
suffix the build is the stock reference, bit for bit.
GPU: unmodified input scripts run with "-sf b200" end in the same atom state
as the reference's own run, bit for bit.
"""
import json
import os

import numpy as np
import pytest

import ref
from ref_scenes import SCENES, digest_dump, first_difference

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_digests.json")
with open(GOLDEN) as _f:
    DIGESTS = json.load(_f)


def _b200_build():
    try:
        return ref.build_b200()
    except Exception:
        return False


def _run_b200(sc, segments, edit=None, suffix=True):
    """The scene's input script through the b200 build; `edit` rewrites lines."""
    def lines(wd):
        ls = ref.script(sc, wd, segments, ["s%d" % i for i in range(len(segments))])
        return edit(ls) if edit else ls
    return ref.run(sc, segments, harness=ref.HARNESS_B200, extra_args=["-sf", "b200"] if suffix else [],
                   script_lines=lines)


def _screen_error(exc):
    msg = str(exc)
    i = msg.find("ERROR")
    return msg[i:i + 400] if i >= 0 else msg[-400:]


@pytest.fixture(scope="module")
def b200():
    if not _b200_build():
        pytest.skip("b200 build of the reference not available (needs the reference sources)")
    return True


def test_unsuffixed_b200_build_is_the_reference(b200):
    """Adding the styles changes nothing for scripts that do not select them."""
    build, segments = SCENES["pour3k_rolling"]
    sc = build()
    got = [digest_dump(sc, d) for d in _run_b200(sc, segments, suffix=False)]
    for w, g in zip(DIGESTS["pour3k_rolling"]["checkpoints"], got):
        assert first_difference(w, g) is None


@pytest.mark.parametrize("edit,expect", [
    (lambda ls: [l.replace("model hertz tangential history", "model hooke tangential history")
                 if l.startswith("pair_style") else l for l in ls], "pair_style gran/b200: 'model hooke'"),
    (lambda ls: [l + " store_force yes" if l.startswith("fix f1 all wall/gran") else l for l in ls],
     "fix wall/gran/b200: 'store_force"),
    (lambda ls: ls[:-4] + ["fix visc all viscous 0.1"] + ls[-4:], "fix visc (style viscous) is outside"),
    (lambda ls: [l.split(" vector")[0] + " spherical 0 180" if " gravity " in l else l for l in ls],
     "fix gravity/b200: only"),
])
def test_suffix_rejects_what_is_off_the_path(b200, edit, expect):
    sc = SCENES["pour3k_rolling"][0]()
    with pytest.raises(RuntimeError) as ei:
        _run_b200(sc, [0, 10], edit=edit)
    assert expect in str(ei.value), _screen_error(ei.value)


def test_suffix_selects_the_device_integrator(b200):
    """With -sf b200 the default run_style becomes verlet/b200, whose setup
    builds the device context (on a host without a B200 it stops there)."""
    import granb200
    sc = SCENES["pour3k_rolling"][0]()
    try:
        _run_b200(sc, [0, 10])
    except RuntimeError as e:
        assert "run_style verlet/b200: no usable B200" in str(e), _screen_error(e)
        return
    # a device is present: the run went through verlet/b200 (checked on the GPU)
    assert granb200.lib() is not None


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["pour3k_rolling", "two_types_schedule", "hopper_mesh", "drum_rotating",
                                  "silo_cylinder_piston", "hopper_packed_discharge"])
def test_suffix_run_equals_reference(b200, name):
    """An unmodified input script with -sf b200: at every checkpoint (each a
    separate 'run N pre no post no', the device context carried across) the
    atoms (x, v, omega, f, torque in local order) equal the reference's run."""
    build, segments = SCENES[name]
    sc = build()
    dumps = _run_b200(sc, segments)
    want = DIGESTS[name]["checkpoints"]
    for k, (w, d) in enumerate(zip(want, dumps)):
        g = digest_dump(sc, d)
        assert g["atoms"] == w["atoms"], "%s: atoms differ from the reference at step %d" % (name, w["ntimestep"])
        assert g["nlocal"] == w["nlocal"]


@pytest.mark.gpu
@pytest.mark.parametrize("name,nseg", [("hopper_mesh", 3), ("drum_rotating", 6)])
def test_suffix_histories_written_back(b200, name, nseg):
    """After a -sf b200 run the reference's own fixes hold the device's
    state: a following 'run 0' (a CPU setup from the written-back pair
    partner arrays, primitive-wall history, mesh contact slots and moved mesh
    nodes) gives the reference's state bit for bit -- atoms, the rebuilt pair
    list with its contact flags and shear history, wall history and mesh
    contacts."""
    build, segments = SCENES[name]
    sc = build()
    segs = segments[:nseg]

    def lines(wd):
        ls = ref.script(sc, wd, segs, ["s%d" % i for i in range(len(segs))])
        return ls + ["run 0", "#@dump s%d" % len(segs)]
    b = ref.run(sc, segs + [0], harness=ref.HARNESS_B200, extra_args=["-sf", "b200"], script_lines=lines)[-1]
    r = ref.run(sc, segs + [0], script_lines=lines)[-1]
    assert np.array_equal(b["tag"], r["tag"])
    for k in ("x", "v", "omega", "f", "torque"):
        assert np.array_equal(b[k], r[k]), k
    for k in ("pair_i", "pair_j", "pair_flag", "pair_hist"):
        assert np.array_equal(b[k], r[k]), k
    assert int((r["pair_flag"] != 0).sum()) > 50
    walls = [k for k in r if k.startswith("w") and k.endswith("_hist")]
    for k in walls:
        assert np.array_equal(b[k], r[k]), k
    for k in ("w0_tag", "w0_tri", "w0_nodes", "w0_vnode"):
        if k in r:
            assert np.array_equal(b[k], r[k]), k
    assert len(r["w0_tag"]) > 0
