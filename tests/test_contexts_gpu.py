"""Many contexts in one process (GPU).

Each context takes its small page-locked words (flags and counts read back
from the device) from a process-wide pinned arena of 256-slot blocks.  These
tests hold more live contexts than one block has slots, and create and
destroy contexts from several host threads at once; every context must
still run the same steps to the same bits.
"""
import threading

import numpy as np
import pytest

import gb2_scenarios as S

pytestmark = pytest.mark.gpu


def _run(sc, steps):
    import granb200
    e = granb200.Engine(sc, device=0)
    try:
        e.setup()
        e.run(steps)
        return e.atoms()
    finally:
        e.close()


def test_more_live_contexts_than_one_arena_block():
    import granb200
    sc = S.sphere_pour(n=300, seed=4)
    ref = _run(sc, 20)
    live = [granb200.Engine(sc, device=0) for _ in range(300)]   # one block holds 256 slots
    try:
        for e in live[::37] + live[-3:]:
            e.setup()
            e.run(20)
            a = e.atoms()
            for k in ("x", "v", "omega", "f", "torque"):
                assert np.array_equal(a[k], ref[k]), k
    finally:
        for e in live:
            e.close()


def test_contexts_created_from_several_threads():
    sc = S.sphere_pour(n=300, seed=5)
    ref = _run(sc, 20)
    errors = []

    def worker():
        try:
            for _ in range(12):
                a = _run(sc, 20)
                for k in ("x", "v", "omega", "f", "torque"):
                    if not np.array_equal(a[k], ref[k]):
                        errors.append(k)
        except Exception as exc:   # reported by the main thread
            errors.append(repr(exc))

    threads = [threading.Thread(target=worker) for _ in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
