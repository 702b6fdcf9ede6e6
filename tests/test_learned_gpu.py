"""The learned split on the GPU: the tensor-core forward and backward match
the CPU restatement (oracle/mlp_ref.py) within bf16 tolerance; training
lowers the loss; builds that start from predicted brackets -- verified or
failed -- give the same tables as the plain build and the oracle; and the
trained network resolves key bits that the plain select would spend digit
passes on."""
import numpy as np
import pytest

import fkdtree_b200 as F
from fkdtree_b200 import workloads as W
from oracle import mlp_ref as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rand_params(seed, scale=0.25):
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(R.NPARAM) * scale).astype(np.float32)
    p[R.OFF_W1 + R.IN * R.H:R.OFF_B1] = 0.0
    return p


def test_forward_matches_reference(cuda):
    m = F.MLP(seed=1)
    p = rand_params(2)
    m.params = p
    x = np.random.default_rng(3).standard_normal((1000, R.IN)).astype(np.float32)
    y = m.forward(x)
    yr, _ = R.forward(p, x)
    np.testing.assert_allclose(y, yr, rtol=2e-3, atol=2e-3)


def test_gradient_matches_reference(cuda):
    m = F.MLP(seed=1)
    p = rand_params(4)
    m.params = p
    rng = np.random.default_rng(5)
    x = rng.standard_normal((333, R.IN)).astype(np.float32)  # not a multiple of the 16-row tiles
    t = rng.standard_normal(333).astype(np.float32)
    g, loss = m.grad(x, t)
    gr, lr = R.grad(p, x, t)
    assert abs(loss - lr) <= 1e-3 * abs(lr) + 1e-5
    assert np.all(g[R.OFF_W1 + R.IN * R.H:R.OFF_B1] == 0.0)
    # bf16-rounded intermediates can flip by one bf16 ulp where the GPU's fp32
    # and the reference's fp64 sums differ in the last bits: compare blocks
    # by relative norm and elements with a bf16-sized tolerance
    for a, b in [(R.OFF_W1, R.OFF_B1), (R.OFF_B1, R.OFF_W2), (R.OFF_W2, R.OFF_B2), (R.OFF_B2, R.OFF_W3),
                 (R.OFF_W3, R.OFF_B3), (R.OFF_B3, R.NPARAM)]:
        ga, gb = g[a:b].astype(np.float64), gr[a:b]
        assert np.linalg.norm(ga - gb) <= 1e-2 * np.linalg.norm(gb) + 1e-7, (a, b)
        np.testing.assert_allclose(ga, gb, rtol=3e-2, atol=3e-2 * np.abs(gb).max() + 1e-7)


def test_training_lowers_the_loss(cuda):
    rng = np.random.default_rng(6)
    x = rng.standard_normal((4096, R.IN)).astype(np.float32)
    t = (0.5 + 0.2 * np.tanh(x[:, 8] - x[:, 9] + 0.5 * x[:, 3])).astype(np.float32)
    m = F.MLP(seed=7)
    losses = m.train(x, t, epochs=25, batch=256, lr=3e-3)
    assert losses[-1] < 0.25 * losses[0]


def _batch(n_events, seed):
    return W.event_batch(n_events=n_events, median=20_000, size_lo=1_000, size_hi=200_000, clusters_lo=50,
                         clusters_hi=500, half_width=0.01, seed=seed, queries=False)


def test_learned_builds_are_bit_identical_and_save_passes(cuda):
    train = _batch(96, 10)
    b = F.Batch.of(train)
    x, t = b.record(train.coords, train.ids)
    assert x.shape[0] > 200
    m = F.MLP(seed=11)
    losses = m.train(x, t, epochs=40, batch=128, lr=2e-3)
    assert losses[-1] < losses[0]
    ev = _batch(48, 20)
    otab, otid, _, _ = O.batch(ev)
    eb = F.Batch.of(ev)
    eb.learn_stats(reset=True)
    eb.build(ev.coords, ev.ids)
    plain = eb.learn_stats(reset=True)
    tab0, tid0 = eb.tables()
    assert np.array_equal(tab0.view(np.uint32), otab.view(np.uint32)) and np.array_equal(tid0, otid)
    assert plain["brackets"] == 0 and plain["passes"] > 0
    eb.set_mlp(m, delta=0.1)
    eb.build(ev.coords, ev.ids)
    tab1, tid1 = eb.tables()
    st = eb.learn_stats(reset=True)
    assert np.array_equal(tab1.view(np.uint32), otab.view(np.uint32)) and np.array_equal(tid1, otid)
    assert st["brackets"] > 0 and st["verified"] + st["fallbacks"] == st["brackets"]
    # what the trained network gains: a verified bracket is binned instead of
    # the node's whole value range, so fewer candidates are left after the
    # first pass and the select needs fewer digit passes than without the
    # network -- and fewer than with an untrained network, whose brackets
    # (around a guess near the middle of the node's range) mostly miss and
    # cost a pass each
    untrained = F.MLP(seed=99)
    eb.set_mlp(untrained, delta=0.1)
    eb.build(ev.coords, ev.ids)
    su = eb.learn_stats(reset=True)
    tab2, tid2 = eb.tables()
    assert np.array_equal(tab2.view(np.uint32), otab.view(np.uint32)) and np.array_equal(tid2, otid)
    assert st["verified"] >= 0.6 * st["brackets"], st
    assert st["verified"] > su["verified"]
    assert st["passes"] < plain["passes"], (st, plain)
    assert st["passes"] < su["passes"], (st, su)


def test_wrong_predictions_fall_back_exactly(cuda):
    """A network that predicts the top of every node's sample range (b3 = 1,
    every other parameter 0) brackets a value far above nearly every split;
    those brackets fail and the plain select takes over: the same tree.  A
    prediction outside the node's value range makes no bracket at all
    (b3 = 50)."""
    ev = _batch(24, 30)
    otab, otid, _, _ = O.batch(ev)
    m = F.MLP(seed=1)
    p = np.zeros(m.n_params, dtype=np.float32)
    p[R.OFF_B3] = 1.0
    m.params = p
    eb = F.Batch.of(ev).set_mlp(m, delta=0.01)
    eb.build(ev.coords, ev.ids)
    tab, tid = eb.tables()
    st = eb.learn_stats(reset=True)
    assert np.array_equal(tab.view(np.uint32), otab.view(np.uint32)) and np.array_equal(tid, otid)
    assert st["brackets"] > 0 and st["verified"] + st["fallbacks"] == st["brackets"]
    assert st["fallbacks"] >= 0.9 * st["brackets"], st
    p[R.OFF_B3] = 50.0
    m.params = p
    eb.set_mlp(m, delta=0.01)
    eb.build(ev.coords, ev.ids)
    tab, tid = eb.tables()
    st = eb.learn_stats(reset=True)
    assert np.array_equal(tab.view(np.uint32), otab.view(np.uint32)) and np.array_equal(tid, otid)
    assert st["brackets"] == 0


def test_learned_single_event_build(cuda):
    ev = W.clustered_event(n=1 << 20, n_queries=1, n_clusters=256, seed=12)
    t = F.FKDTree(ev.coords, ev.ids)
    m = F.MLP(seed=3)
    t.set_mlp(m, delta=0.2)
    t.build()
    assert_tab = O.build(ev.coords, ev.ids)
    tab, tid = t.tables()
    assert np.array_equal(tab.view(np.uint32), assert_tab[0].view(np.uint32)) and np.array_equal(tid, assert_tab[1])
    st = t.learn_stats()
    assert st["verified"] + st["fallbacks"] == st["brackets"]
