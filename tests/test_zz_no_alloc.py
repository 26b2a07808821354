"""gb2_census_noalloc -- the census entry point for callers that cannot
allocate device memory (a monitoring hook inside a framework whose pool owns
every device allocation, or a process at its device-memory cap).  Its
scratch is a static device array inside libgranb200, so its counts must
equal those of the allocating gb2_census, call after call.  (A context with
no atoms, answered with zeros before any launch, cannot be built through the
ABI: gb2_upload_atoms needs at least one atom.)

This file is collected last so that a failure here cannot hide the result of
any other test in a run that stops at the first failure.
"""
import pytest

import gb2_scenarios as S

pytestmark = pytest.mark.gpu


def _engine(sc, steps):
    import granb200
    e = granb200.Engine(sc)
    e.setup()
    e.run(steps)
    return e


def test_noalloc_census_matches_allocating_census():
    sc = S.hopper(n=20000, n_theta=48, n_z=12, seed=8, gap=0.01, vmax=0.05)
    e = _engine(sc, 300)
    ref = e.census()
    assert ref["nlist"] > 0 and ref["ntouch"] > 0 and ref["nmesh_cand"] > 0
    for _ in range(2):                      # two calls in a row share the static scratch
        assert e.census_noalloc() == ref
    e.run(50)                               # state changes, counts must follow it
    ref2 = e.census()
    for _ in range(2):
        assert e.census_noalloc() == ref2


def test_noalloc_census_second_context_same_device():
    sc = S.sphere_pour(n=3000, seed=2)
    a = _engine(sc, 200)
    b = _engine(S.hopper(n=5000, n_theta=32, n_z=8, seed=3, gap=0.01, vmax=0.05), 100)
    for e in (a, b, a, b):
        assert e.census_noalloc() == e.census()


def test_noalloc_census_rejects_oversize_context():
    import granb200
    n = granb200.NOALLOC_MAX_ATOMS + 1000
    sc = S.hopper(n=n, seed=1, gap=0.01)
    e = _engine(sc, 0)
    with pytest.raises(granb200.GB2Error, match="at most"):
        e.census_noalloc()
    assert e.census()["nlist"] > 0          # the allocating census still serves it
