"""The per-environment bridge: ragged sequences of per-environment solve
calls become one solve_batch per round, environments run one at a time in
order, rows come back to their callers, errors propagate (CPU, with a
HiGHS-backed stand-in for the batched backend)."""

from types import SimpleNamespace

import numpy as np
import pytest
from scipy.optimize import linprog

from co_cultivation_metabolic_atlas_b200.bridge import BatchingBridge


class HighsBatch:
    name = "highs_batch"
    method = "highs"

    def __init__(self):
        self.calls = []

    def solve_batch(self, requests, *, environment_ids=None):
        self.calls.append(list(environment_ids))
        rows = []
        for c, kw in requests:
            kw = {k: v for k, v in kw.items() if not k.startswith("_")}
            r = linprog(c, **kw)
            rows.append(SimpleNamespace(success=r.status == 0, x=r.x, fun=r.fun, message=r.message,
                                        diagnostics=dict(environment=len(rows))))
        return rows


def lp(k):
    """min -x0 - k x1  s.t.  x0 + x1 <= 1 + k,  0 <= x <= 2."""
    return (np.array([-1.0, -float(k)]), dict(A_ub=np.array([[1.0, 1.0]]), b_ub=np.array([1.0 + k]),
                                              bounds=[(0, 2), (0, 2)], method="highs"))


def test_ragged_rounds_sequential_turns_and_rows():
    parent = HighsBatch()
    bridge = BatchingBridge(parent)
    trace = []
    calls = {0: 1, 1: 2, 2: 3, 3: 1, 4: 2}

    def make(env):
        def fn(backend):
            out = []
            for q in range(calls[env]):
                trace.append((env, q))
                c, kw = lp(env + q)
                out.append(backend.solve(c, **kw).fun)
            assert len(backend.history) == calls[env]
            return out
        return fn

    res = bridge.run({env: make(env) for env in calls})
    assert bridge.rounds == [5, 3, 1]
    assert parent.calls == [[0, 1, 2, 3, 4], [1, 2, 4], [2]]
    # one environment at a time, in order, each up to its next solve
    assert trace == [(0, 0), (1, 0), (2, 0), (3, 0), (4, 0), (1, 1), (2, 1), (4, 1), (2, 2)]
    for env, funs in res.items():
        for q, f in enumerate(funs):
            c, kw = lp(env + q)
            assert f == pytest.approx(linprog(c, **kw).fun)


def test_environment_errors_and_backend_errors_propagate():
    parent = HighsBatch()
    bridge = BatchingBridge(parent)

    def bad(backend):
        backend.solve(*lp(1)[:1], **lp(1)[1])
        raise KeyError("environment failure")

    def good(backend):
        return backend.solve(*lp(2)[:1], **lp(2)[1]).fun

    with pytest.raises(KeyError):
        bridge.run({"a": bad, "b": good})

    class Broken(HighsBatch):
        def solve_batch(self, requests, *, environment_ids=None):
            raise ValueError("backend failure")

    with pytest.raises(ValueError, match="backend failure"):
        BatchingBridge(Broken()).run({"a": good, "b": good})
    with pytest.raises(ValueError):
        BatchingBridge(object())
