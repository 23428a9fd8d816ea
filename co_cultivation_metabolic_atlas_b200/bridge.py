"""Per-environment ``solve(c, **kwargs)`` calls gathered into batched solves.

The reference runs each environment's step code (for instance its
cooperative solver, which calls ``linear_program_backend.solve(objective,
**kwargs)`` once per stage) as a greenlet and hands every environment a
``YieldingLPBackend`` whose ``solve`` switches to the driver; the driver
collects one request per environment and answers them all with one
``solve_batch`` (``src/gpu_batched_compiled_backend.py:532-542``).

``BatchingBridge`` keeps that contract without greenlets.  Each
environment's code runs in its own thread with a per-environment backend
(``name``, ``method``, ``history``, ``solve(c, **kwargs)``), but only one of
them runs at a time, as with greenlets: the driver gives each environment in
turn the right to run until it calls ``solve`` (its request joins the round)
or returns; when every environment has had its turn, one
``solve_batch(requests, environment_ids=...)`` of the parent backend answers
the round, and the environments that asked continue, in order, with their
rows.  Rounds repeat until every environment has returned.  An exception
raised by an environment's code, or by the batched solve, is re-raised by
``run`` after every thread has stopped.
"""

from __future__ import annotations

import threading


class _EnvironmentBackend:
    """The per-environment face of the bridge (the ``YieldingLPBackend``
    contract)."""

    def __init__(self, bridge, environment_id):
        self._bridge = bridge
        self.environment_id = environment_id
        self.name = getattr(bridge.parent, "name", "batching_bridge")
        self.method = getattr(bridge.parent, "method", "")
        self.history: list[dict] = []

    def solve(self, c, **kwargs):
        row = self._bridge._submit(self.environment_id, (c, kwargs))
        self.history.append(dict(getattr(row, "diagnostics", {}) or {}))
        return row


class BatchingBridge:
    def __init__(self, parent):
        if not hasattr(parent, "solve_batch"):
            raise ValueError("the parent backend must provide solve_batch")
        self.parent = parent
        self.rounds: list[int] = []      # batch size of every solve_batch call
        self._cv = threading.Condition()
        self._turn = None                # the environment allowed to run
        self._pending: dict = {}
        self._rows: dict = {}
        self._error: BaseException | None = None

    def backend(self, environment_id):
        return _EnvironmentBackend(self, environment_id)

    # -- inside environment threads ------------------------------------------
    def _submit(self, env, request):
        with self._cv:
            if self._error is not None:
                raise RuntimeError("the batched solve failed") from self._error
            self._pending[env] = request
            self._turn = None                    # hand the turn back
            self._cv.notify_all()
            while not (self._turn == env and env in self._rows) and self._error is None:
                self._cv.wait()
            if env not in self._rows:
                raise RuntimeError("the batched solve failed") from self._error
            return self._rows.pop(env)

    def _body(self, env, fn, backend, results, errors):
        with self._cv:
            while self._turn != env and self._error is None:
                self._cv.wait()
        try:
            if self._error is None:
                results[env] = fn(backend)
        except BaseException as exc:  # re-raised by the driver
            errors[env] = exc
        finally:
            with self._cv:
                self._turn = None
                self._cv.notify_all()

    # -- driver ----------------------------------------------------------------
    def _give_turns(self, envs):
        for env in envs:
            with self._cv:
                self._turn = env
                self._cv.notify_all()
                while self._turn is not None:
                    self._cv.wait()

    def run(self, functions):
        """Run ``functions[env](backend)`` for every environment id (in the
        mapping's order) and return ``{env: return value}``; each function
        receives its per-environment backend."""
        functions = dict(functions)
        order = list(functions)
        results, errors = {}, {}
        with self._cv:
            self._turn = None
            self._pending.clear()
            self._rows.clear()
            self._error = None
        threads = [threading.Thread(target=self._body, args=(env, functions[env], self.backend(env), results, errors),
                                    daemon=True) for env in order]
        for t in threads:
            t.start()
        active = order
        try:
            while True:
                self._give_turns(active)
                with self._cv:
                    if not self._pending:
                        break
                    ids = [e for e in order if e in self._pending]
                    requests = [self._pending.pop(e) for e in ids]
                rows = self.parent.solve_batch(requests, environment_ids=ids)
                if len(rows) != len(ids):
                    raise RuntimeError("solve_batch returned the wrong number of rows")
                with self._cv:
                    self.rounds.append(len(ids))
                    self._rows.update(zip(ids, rows))
                active = ids
        except BaseException as exc:
            with self._cv:
                self._error = exc
                self._turn = None
                self._cv.notify_all()
            for t in threads:
                t.join()
            raise
        for t in threads:
            t.join()
        if errors:
            raise next(iter(errors.values()))
        return results
