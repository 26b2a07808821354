"""Regenerate reference_digests.json from the reference itself.

Runs every scene of tests/ref_scenes.py (the restart scenes through a real
restart file) through the reference harness
(oracle/_ref/ref_harness, built from the reference's sources by
oracle/Makefile.ref) and writes, per checkpoint, SHA-256 digests of the raw
state: atoms (tag, x, v, omega, f, torque in local order), the pair list
(tags, contact flags, shear history in list order), every wall's contact
history and mesh nodes / node velocities, plus counts.  The tests compare
the oracle and the engine against these digests, so they need no reference
build at run time.

    python tests/golden/make_golden.py [scene ...]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("oracle", os.path.join("liggghts-public_b200", "python"), "tests"):
    sys.path.insert(0, os.path.join(ROOT, sub))

import ref  # noqa: E402
import ref_scenes  # noqa: E402

OUT = os.path.join(HERE, "reference_digests.json")


def main(names):
    if not ref.build():
        raise SystemExit("the reference harness is not built and its sources are absent")
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for name in names or list(ref_scenes.ALL_SCENES) + list(ref_scenes.RESTART_SCENES):
        t = time.time()
        if name in ref_scenes.RESTART_SCENES:
            build, n_before, segments = ref_scenes.RESTART_SCENES[name]
            sc = build()
            dumps = ref.run_restart(sc, n_before, segments)
            data[name] = {"restart_after": n_before, "segments": segments,
                          "checkpoints": [ref_scenes.digest_dump(sc, d) for d in dumps]}
        else:
            build, segments = ref_scenes.ALL_SCENES[name]
            sc = build()
            dumps = ref.run(sc, segments)
            data[name] = {"segments": segments, "checkpoints": [ref_scenes.digest_dump(sc, d) for d in dumps]}
        print("%-32s %6.1f s  last: %s" % (name, time.time() - t, {k: v for k, v in data[name]["checkpoints"][-1].items()
                                                                     if not isinstance(v, str)}))
    data = {k: data[k] for k in sorted(data)}
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:])
