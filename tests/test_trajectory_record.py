"""The committed log-likelihood trajectory record of the 60M-token corpus
(profiles/trajectory_plain-cgs-scale.json, made on a B200 by
tests/trajectory/make_trajectory.py): the reference's own build over five
runs against this library over five seeds, 100 iterations each.

The per-checkpoint summary must follow from the series.  What the record
shows is checked as it stands: this library's states, scored by the
reference's own printed formula (the oracle's restatement of it), are within
0.5% of the reference's printed values at iteration 10 and never worse than
them by more than 0.5% at any checkpoint; later the gap grows the other way
(this chain's log-likelihood rises faster per iteration), so the 0.5% window
is not met there, and this library reaches the reference's iteration-100 value
in well under 100 iterations.
"""
from __future__ import annotations

import json
import statistics
from pathlib import Path

import pytest

RECORD = Path(__file__).resolve().parents[1] / "profiles" / "trajectory_plain-cgs-scale.json"
WINDOW = 0.005  # relative, of the reference's value


@pytest.fixture(scope="module")
def rec():
    return json.loads(RECORD.read_text())


def _mean_series(runs):
    n = len(runs[0]["loglik"])
    return [statistics.mean(r["loglik"][i] for r in runs) for i in range(n)]


def test_record_holds_every_series(rec):
    it, runs = rec["iterations"], rec["runs"]
    assert it >= 100 and runs >= 5
    assert len(rec["reference"]) == runs and len(rec["ours"]) == runs
    assert all(len(x["loglik"]) == it for x in rec["reference"] + rec["ours"])
    assert sorted(x["seed"] for x in rec["ours"]) == list(range(1, runs + 1))
    assert rec["num_tokens"] > 60_000_000 and rec["k"] == 1024


def test_summary_follows_from_the_series(rec):
    for row in rec["checkpoints"]:
        i = row["iteration"]
        r = [x["loglik"][i - 1] for x in rec["reference"]]
        o = [x["loglik"][i - 1] for x in rec["ours"]]
        f = [x["loglik_reference_formula"][str(i)] for x in rec["ours"]]
        assert row["reference_mean"] == pytest.approx(statistics.mean(r), rel=1e-12)
        assert row["ours_mean"] == pytest.approx(statistics.mean(o), rel=1e-12)
        assert row["ours_reference_formula_mean"] == pytest.approx(statistics.mean(f), rel=1e-12)
        gap = 100.0 * (statistics.mean(f) - statistics.mean(r)) / abs(statistics.mean(r))
        assert row["gap_pct_reference_formula"] == pytest.approx(gap, abs=1e-9)
        assert row["within_0_5pct_reference_formula"] == (abs(gap) <= 100 * WINDOW)


def test_every_chain_improves(rec):
    for x in rec["reference"] + rec["ours"]:
        assert x["loglik"][99] > x["loglik"][9] > x["loglik"][0]


def test_window_at_iteration_10_and_never_worse_than_the_reference(rec):
    rows = {row["iteration"]: row for row in rec["checkpoints"]}
    assert rows[10]["within_0_5pct_reference_formula"]
    for row in rows.values():
        assert row["gap_pct_reference_formula"] >= -100 * WINDOW


def test_this_chain_reaches_the_reference_iteration_100_value_sooner(rec):
    ours, ref = _mean_series(rec["ours"]), _mean_series(rec["reference"])
    first = next(i + 1 for i, v in enumerate(ours) if v >= ref[99])
    assert first < 100
