"""Host logic of the drop-in's learned warm start (no GPU): feature
selection, and the propose/commit transaction over per-environment
histories (``src/temporal_lp_model.py:221-285`` semantics)."""
import numpy as np

from co_cultivation_metabolic_atlas_b200.warmstart import RequestWarmStart, select_request_features, signed_log


class FakeEngine:
    def __init__(self, shapes):
        self.shapes = shapes  # (m, n) per species

    def layout(self, species):
        n = np.array([self.shapes[s][1] for s in species])
        m = np.array([self.shapes[s][0] for s in species])
        co = np.concatenate([[0], np.cumsum(n)[:-1]])
        ro = np.concatenate([[0], np.cumsum(m)[:-1]])
        return co, ro, int(n.sum()), int(m.sum())


def problem(n, m, lo=0.0):
    return (None, np.zeros(m), np.full(n, lo), np.full(n, 10.0), np.ones(n), m)


def test_signed_log_and_feature_selection():
    assert signed_log([0.0, np.e - 1, -(np.e - 1), np.inf])[:3].tolist() == [0.0, 1.0, -1.0]
    rng = np.random.default_rng(0)
    base = rng.normal(size=(50, 1))
    full = np.concatenate([np.ones((50, 3)), base, base, rng.normal(size=(50, 200))], axis=1)
    idx = select_request_features(full, limit=128)
    assert 0 not in idx and not (3 in idx and 4 in idx)  # constants dropped, duplicates collapsed
    assert idx.size == 128 and np.all(np.diff(idx) > 0)
    assert select_request_features(np.ones((5, 4))).tolist() == [0]


def test_propose_is_pending_until_commit_and_failures_clear_history():
    ws = RequestWarmStart({})
    eng = FakeEngine([(2, 3)])
    probs = [problem(3, 2), problem(3, 2)]
    species = np.zeros(2, np.int32)
    keys = ["k", "k"]
    wx, wy, wo = ws.propose(["a", "b"], probs, species, eng, keys=keys)
    assert not wx.any() and ws.last_sources == ["cold", "cold"]
    # a call that raised never commits: the history stays empty
    ws.propose(["a", "b"], probs, species, eng, keys=keys)
    assert ws.last_sources == ["cold", "cold"]
    ws.commit(["a", "b"], {"a": (np.full(3, 1.0), np.full(2, -1.0), 2.0)}, keys)
    wx, wy, wo = ws.propose(["a", "b"], probs, species, eng, keys=keys)
    assert ws.last_sources == ["temporal", "cold"]
    assert wx[:3].tolist() == [1.0] * 3 and wy[:2].tolist() == [-1.0] * 2 and wo.tolist() == [2.0, 1.0]
    # two committed solutions: linear extrapolation
    ws.commit(["a"], {"a": (np.full(3, 1.5), np.full(2, -2.0), 3.0)}, ["k"])
    wx, wy, wo = ws.propose(["a"], probs[:1], species[:1], eng, keys=["k"])
    assert wx.tolist() == [2.0] * 3 and wy.tolist() == [-3.0] * 2 and wo.tolist() == [3.0]
    # a failed row clears its environment; reset clears the rest
    ws.commit(["a"], {}, ["k"])
    ws.propose(["a"], probs[:1], species[:1], eng, keys=["k"])
    assert ws.last_sources == ["cold"]
    ws.commit(["b"], {"b": (np.zeros(3), np.zeros(2), 1.0)}, ["k"])
    ws.reset(["b"])
    ws.propose(["b"], probs[:1], species[:1], eng, keys=["k"])
    assert ws.last_sources == ["cold"]


def test_history_of_another_matrix_is_not_proposed():
    ws = RequestWarmStart({})
    eng = FakeEngine([(2, 3)])
    ws.commit(["a"], {"a": (np.ones(3), np.ones(2), 1.0)}, ["k1"])
    ws.propose(["a"], [problem(3, 2)], np.zeros(1, np.int32), eng, keys=["k2"])
    assert ws.last_sources == ["cold"]
