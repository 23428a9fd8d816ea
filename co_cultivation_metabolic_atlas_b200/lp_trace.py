"""Lossless LP traces: the reference's ``.npz`` trace format and manifest
entries (``src/lp_trace.py:18-96``), so traces captured from the reference's
CPU-HiGHS runs can be replayed through this engine and the engine's own
certified solves can be exported as golden data.

A trace file holds one normalised problem ``(a, rhs, lower, upper, c, neq)``
(CSR arrays ``a_data``, ``a_indices``, ``a_indptr``, ``a_shape``) and a
reference primal/dual pair (``reference_x``, ``reference_y``).  Its manifest
entry carries the file's sha256, the problem's content hash, its dimensions
and, optionally, ``step`` / ``stage`` / ``environment_id`` labels that must
agree with the file name ``lp_{step:03d}_{stage index}_{env:03d}.npz``.
Loading re-validates everything the way the reference does: the path stays
inside the trace directory, the checksum matches, the problem survives a
round trip through the request normaliser unchanged, the labels agree, and
the reference solution passes the original-LP certificate gate.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
from scipy.sparse import csr_matrix

from .problem import normalize, request

STAGES = ("maxmin", "aggregate", "exchange")
PRIMAL_GATE, DUAL_GATE, GAP_GATE = 1e-5, 1e-7, 1e-7  # src/gpu_block_lp.py:84


def problem_hash(problem) -> str:
    """Content hash of a normalised problem (same field order, names and
    little-endian encodings as the reference's ``problem_hash``, so hashes
    recorded by the reference are reproduced)."""
    a, rhs, lower, upper, c, neq = problem
    digest = hashlib.sha256()
    for name, value in (("shape", a.shape), ("data", a.data), ("indices", a.indices), ("indptr", a.indptr),
                        ("rhs", rhs), ("lower", lower), ("upper", upper), ("c", c), ("neq", neq)):
        array = np.asarray(value, dtype="<i8" if name in {"shape", "indices", "indptr", "neq"} else "<f8")
        digest.update(name.encode())
        digest.update(np.asarray(array.shape, dtype="<i8").tobytes())
        digest.update(array.tobytes())
    return digest.hexdigest()


def certificate(problem, x, y) -> dict:
    """Original-LP certificate of a primal/dual pair on the host (input
    validation of traces; the solver's own certificate runs on the GPU):
    primal residual, dual violation and relative KKT gap with the
    reference's gate."""
    a, rhs, lower, upper, c, neq = problem
    x = np.asarray(x, dtype=float)
    y = np.asarray(y, dtype=float)
    if x.shape != c.shape or y.shape != rhs.shape or not (np.isfinite(x).all() and np.isfinite(y).all()):
        return dict(primal_residual=np.inf, dual_violation=np.inf, relative_kkt_gap=np.inf,
                    certificate_passed=False)
    activity = a @ x
    reduced = c - a.T @ y
    err = activity - rhs
    primal = max(0.0, np.max(np.abs(err[:neq]), initial=0.0), np.max(err[neq:], initial=0.0),
                 np.max(lower - x, initial=0.0), np.max(x - upper, initial=0.0))
    dual = max(0.0, np.max(y[neq:], initial=0.0), np.max(np.where(np.isinf(lower), reduced, 0.0), initial=0.0),
               np.max(np.where(np.isinf(upper), -reduced, 0.0), initial=0.0))
    target = np.where(reduced >= 0.0, lower, upper)
    gap = (np.abs(reduced * (x - np.where(np.isfinite(target), target, x))).sum()
           + np.abs(y[neq:] * (rhs - activity)[neq:]).sum()) / max(1.0, abs(float(c @ x)))
    return dict(primal_residual=float(primal), dual_violation=float(dual), relative_kkt_gap=float(gap),
                certificate_passed=bool(primal <= PRIMAL_GATE and dual <= DUAL_GATE and gap <= GAP_GATE))


def trace_filename(step: int, stage: str, environment_id: int) -> str:
    return f"lp_{step:03d}_{STAGES.index(stage)}_{environment_id:03d}.npz"


def write_trace_lp(path, problem, *, reference_x, reference_y) -> dict:
    """Write one trace file (refusing to overwrite) and return its manifest
    entry."""
    path = Path(path)
    if path.exists():
        raise FileExistsError(path)
    a, rhs, lower, upper, c, neq = problem
    x, y = np.asarray(reference_x), np.asarray(reference_y)
    if x.shape != c.shape or y.shape != rhs.shape or not (np.isfinite(x).all() and np.isfinite(y).all()):
        raise ValueError("Invalid reference solution")
    np.savez_compressed(path, a_data=a.data, a_indices=a.indices, a_indptr=a.indptr, a_shape=a.shape, rhs=rhs,
                        lower=lower, upper=upper, c=c, neq=neq, reference_x=x, reference_y=y)
    return dict(filename=path.name, sha256=hashlib.sha256(path.read_bytes()).hexdigest(),
                problem_sha256=problem_hash(problem), rows=a.shape[0], columns=a.shape[1], nonzeros=a.nnz,
                equalities=int(neq))


def load_trace_lp(directory, entry):
    """Load and validate one manifest entry; returns ``(problem, x, y)``.
    Raises ``ValueError`` for anything the reference's loader rejects."""
    directory = Path(directory).resolve()
    path = (directory / entry["filename"]).resolve()
    if not path.is_relative_to(directory) or not path.is_file() or \
            hashlib.sha256(path.read_bytes()).hexdigest() != entry["sha256"]:
        raise ValueError("Untrusted LP trace path or checksum")
    with np.load(path, allow_pickle=False) as data:
        a = csr_matrix((data["a_data"], data["a_indices"], data["a_indptr"]), shape=tuple(data["a_shape"]))
        problem = (a, data["rhs"], data["lower"], data["upper"], data["c"], int(data["neq"]))
        x, y = data["reference_x"], data["reference_y"]
    rebuilt = normalize(*request(problem))
    if problem_hash(rebuilt) != entry["problem_sha256"]:
        raise ValueError("LP trace input changed during restoration")
    a, rhs, _, _, c, neq = rebuilt
    if (entry.get("rows"), entry.get("columns"), entry.get("nonzeros"), entry.get("equalities")) != (
            a.shape[0], a.shape[1], a.nnz, neq):
        raise ValueError("LP trace dimension metadata does not match its payload")
    if any(k in entry for k in ("step", "stage", "environment_id")):
        stage, step, env = entry.get("stage"), entry.get("step"), entry.get("environment_id")
        if stage not in STAGES or not (isinstance(step, int) and step >= 1 and isinstance(env, int) and env >= 0):
            raise ValueError("Invalid LP trace labels")
        if entry["filename"] != trace_filename(step, stage, env):
            raise ValueError("LP trace labels disagree with the recorded filename")
    if x.shape != c.shape or y.shape != rhs.shape or not (np.isfinite(x).all() and np.isfinite(y).all()):
        raise ValueError("Invalid reference solution")
    if not certificate(rebuilt, x, y)["certificate_passed"]:
        raise ValueError("Reference solution does not certify the original LP")
    return rebuilt, x, y


def write_manifest(directory, entries, *, name="manifest.json"):
    """Write the manifest atomically (temporary file, then rename)."""
    directory = Path(directory)
    tmp = directory / (name + ".tmp")
    tmp.write_text(json.dumps({"traces": list(entries)}, indent=1, sort_keys=True))
    tmp.replace(directory / name)


def read_manifest(directory, *, name="manifest.json"):
    return json.loads((Path(directory) / name).read_text())["traces"]


def replay(directory, backend, *, name="manifest.json", environment_ids=None):
    """Solve every trace of a manifest through a ``solve_batch`` backend in
    one batch and compare with the recorded reference objectives.  Returns
    ``(rows, reference_objectives)``."""
    entries = read_manifest(directory, name=name)
    loaded = [load_trace_lp(directory, e) for e in entries]
    requests = [request(p) for p, _, _ in loaded]
    rows = backend.solve_batch(requests, environment_ids=environment_ids)
    ref = [float(p[4] @ x) for p, x, _ in loaded]
    return rows, ref
