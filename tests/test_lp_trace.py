"""LP traces: files and manifest entries written by the reference's own
trace writer load, validate and hash identically here; the engine's writer
round-trips; every tampering the reference rejects is rejected."""
import json
import shutil

import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import lp_trace
from co_cultivation_metabolic_atlas_b200.problem import normalize, request


@pytest.fixture()
def traces(golden_dir, tmp_path):
    d = tmp_path / "traces"
    shutil.copytree(golden_dir / "traces", d)
    return d


def test_reference_written_traces_load_and_hash_identically(traces, golden_dir):
    entries = lp_trace.read_manifest(traces)
    hashes = json.loads((golden_dir / "trace_hashes.json").read_text())
    assert len(entries) == 3
    for e in entries:
        problem, x, y = lp_trace.load_trace_lp(traces, e)
        assert lp_trace.problem_hash(problem) == e["problem_sha256"] == hashes[e["filename"]]
        assert lp_trace.certificate(problem, x, y)["certificate_passed"]
    labelled = [e for e in entries if "stage" in e]
    assert labelled and labelled[0]["filename"] == lp_trace.trace_filename(1, "exchange", 4)


def test_engine_written_trace_round_trips(traces, tmp_path):
    e = lp_trace.read_manifest(traces)[0]
    problem, x, y = lp_trace.load_trace_lp(traces, e)
    out = tmp_path / "mine"
    out.mkdir()
    entry = lp_trace.write_trace_lp(out / "lp_x.npz", problem, reference_x=x, reference_y=y)
    assert entry["problem_sha256"] == e["problem_sha256"]
    with pytest.raises(FileExistsError):
        lp_trace.write_trace_lp(out / "lp_x.npz", problem, reference_x=x, reference_y=y)
    lp_trace.write_manifest(out, [entry])
    back, x2, y2 = lp_trace.load_trace_lp(out, lp_trace.read_manifest(out)[0])
    assert lp_trace.problem_hash(back) == entry["problem_sha256"]
    np.testing.assert_array_equal(x2, x)
    assert lp_trace.problem_hash(normalize(*request(back))) == entry["problem_sha256"]


def test_tampering_is_rejected(traces):
    entries = lp_trace.read_manifest(traces)
    e = dict(entries[0])
    with pytest.raises(ValueError, match="Untrusted"):
        lp_trace.load_trace_lp(traces, dict(e, filename="../" + e["filename"]))
    with pytest.raises(ValueError, match="Untrusted"):
        lp_trace.load_trace_lp(traces, dict(e, sha256="0" * 64))
    with pytest.raises(ValueError, match="changed"):
        lp_trace.load_trace_lp(traces, dict(e, problem_sha256="0" * 64))
    with pytest.raises(ValueError, match="dimension"):
        lp_trace.load_trace_lp(traces, dict(e, rows=e["rows"] + 1))
    lab = [x for x in entries if "stage" in x][0]
    with pytest.raises(ValueError, match="labels"):
        lp_trace.load_trace_lp(traces, dict(lab, environment_id=5))
    with pytest.raises(ValueError, match="labels"):
        lp_trace.load_trace_lp(traces, dict(lab, stage="growth"))
    # a reference solution that does not certify
    problem, x, y = lp_trace.load_trace_lp(traces, e)
    bad = traces / "bad.npz"
    entry = lp_trace.write_trace_lp(bad, problem, reference_x=x + 1.0, reference_y=y)
    with pytest.raises(ValueError, match="certify"):
        lp_trace.load_trace_lp(traces, entry)
