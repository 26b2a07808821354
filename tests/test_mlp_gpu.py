"""Learned initial guess of the superquadric contact solve.

* The device forward/backward kernels (BF16 tensor cores, FP32 accumulation)
  against the NumPy reference with the same rounding points: loss to 1e-4
  relative, gradient to 2e-2 relative L2 and cosine similarity > 0.999
  (BF16 rounding of an activation or delta can flip on the last FP32 bit,
  which moves single gradient entries by a BF16 ulp).
* Training on pairs labelled by the plain solver lowers the loss, and the
  trained guess needs fewer Newton solves and iterations than the plain
  method (homotopy from spheres) at the same convergence tolerance
  (merit < 1e-10, which bounds the angle between the two surface normals by
  1e-5, so two converged points may sit ~1e-5 of the particle size apart);
  the plain method stays the fallback.
* In a simulation the learned guess leaves the contact states and forces as
  they are (to the solver tolerance) and lowers the iteration count.
"""
import numpy as np
import pytest

import gb2_scenarios as S
import mlp_oracle
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    import granb200
    t = granb200.MlpTrainer()
    info = t.make_data(200_000, seed=1)
    t.init(seed=2)
    l0, l1 = t.train(epochs=6, batch=2048, lr=2e-3)
    return t, info, l0, l1


def test_gradient_matches_reference():
    import granb200
    t = granb200.MlpTrainer()
    t.make_data(4096, seed=5)
    t.init(seed=6)
    rng = np.random.default_rng(0)
    n = 300
    samples = np.zeros((n, 22), dtype=np.float32)
    samples[:, :14] = rng.normal(size=(n, 14)).astype(np.float32) * 0.3 + 0.2
    samples[:, 14:18] = rng.normal(size=(n, 4)).astype(np.float32) * 0.2
    P = t.params()
    loss, g = t.grad(samples)
    rloss, rg = mlp_oracle.loss_and_grad(P, samples)
    assert abs(loss - rloss) <= 1e-4 * abs(rloss)
    tr = slice(mlp_oracle.OFF_W1, mlp_oracle.SIZE)
    a, b = g[tr].astype(np.float64), rg[tr].astype(np.float64)
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    print("loss %.6g vs %.6g, grad rel L2 %.3g, cos %.7f" % (loss, rloss, rel, cos))
    assert rel <= 2e-2 and cos > 0.999
    # every layer's block is non-trivial and matches on its own
    for lo, hi in ((mlp_oracle.OFF_W1, mlp_oracle.OFF_B1), (mlp_oracle.OFF_W2, mlp_oracle.OFF_B2),
                   (mlp_oracle.OFF_W3, mlp_oracle.OFF_B3), (mlp_oracle.OFF_W4, mlp_oracle.OFF_B4)):
        x, y = g[lo:hi].astype(np.float64), rg[lo:hi].astype(np.float64)
        assert np.linalg.norm(y) > 0
        assert np.linalg.norm(x - y) <= 3e-2 * np.linalg.norm(y)


def test_training_lowers_loss(trained):
    t, info, l0, l1 = trained
    print("samples %d, plain solver %.2f iterations / %.2f solves per pair, loss %.4f -> %.4f" % (
        info["valid"], info["plain_iters"], info["plain_solves"], l0, l1))
    assert info["valid"] > 100_000
    assert l1 < 0.5 * l0


def test_learned_guess_gain(trained):
    t, info, l0, l1 = trained
    ev = t.evaluate(50_000, seed=99)
    print(ev)
    assert ev["pairs"] > 20_000
    assert ev["learned_fail"] <= ev["plain_fail"]
    assert ev["learned_accepted"] >= 0.8 * ev["pairs"]
    assert ev["learned_solves"] < 0.5 * ev["plain_solves"]
    assert ev["learned_iters"] < ev["plain_iters"]
    assert ev["differ"] <= 0.01 * ev["pairs"]
    assert ev["maxdiff"] <= 2e-3


def test_learned_guess_in_simulation(trained):
    import granb200
    t, info, l0, l1 = trained
    sc = S.sq_packing(n=343, seed=3)
    a, b = granb200.SqEngine(sc), granb200.SqEngine(sc, learned=t.params())
    for e in (a, b):
        e.setup()
        e.run(200)
    pa, pb = a.pairs(), b.pairs()
    assert np.array_equal(pa["tag_i"], pb["tag_i"]) and np.array_equal(pa["tag_j"], pb["tag_j"])
    agree = np.mean(pa["state"] == pb["state"])
    fa, fb = a.atoms()["f"], b.atoms()["f"]
    ca, cb = a.counters(), b.counters()
    print("plain", ca, "learned", cb, "state agreement %.4f" % agree)
    assert agree >= 0.99
    assert np.abs(fa - fb).max() <= 1e-3 * np.abs(fa).max()
    assert cb["learned_used"] > 0
    assert cb["solves"] < ca["solves"]


def test_learned_guess_solve_time(trained):
    """The first-contact solve itself on the same fresh pairs both ways: the
    learned guess needs about half the Newton iterations.  The times are
    reported, not asserted (the learned method is its attempts, then the
    homotopy over the pairs it rejected; both launches depend on their
    slowest pairs, which the plain solver may also fail on)."""
    t, info, l0, l1 = trained
    ts = t.time_solves(100_000, seed=7)
    print(ts)
    assert ts["pairs"] > 40_000
    assert ts["learned_iters"] < 0.6 * ts["plain_iters"]
    assert ts["plain_ms"] > 0 and ts["learned_ms"] > 0
