"""The committed autotuner record (treegeneralizedharmonic.jl_b200/tuning/nvidia_b200.json) read on
the CPU: every configuration's choice is the fastest entry of its own sweep, the sweep holds every
candidate the tuner times for that configuration, and GHProblem's lookup returns the choice (and
refuses a TMA choice for a configuration the TMA kernel does not cover)."""
import json
import re
from types import SimpleNamespace

import pytest

from conftest import PKG

RECORD = PKG / "tuning" / "nvidia_b200.json"
KEY = re.compile(r"^q(\d)_n(\d+)_(fp64|mixed)_(interior|nointerior)$")


def _fake_problem(key):
    q, n, precision, interior = KEY.match(key).groups()
    return SimpleNamespace(q=int(q), forest=SimpleNamespace(N=int(n)), precision=precision,
                           case=SimpleNamespace(interior={"variant": "damped"} if interior == "interior" else None))


def _variant(r):
    return (r["pi"], r["threads"], r["pi_mb"])


def test_record_choices_are_the_fastest_of_their_sweeps(tgh):
    at = tgh.autotune
    data = json.loads(RECORD.read_text())
    assert data, "the record is empty"
    for key, rec in data.items():
        assert KEY.match(key), key
        P = _fake_problem(key)
        assert at.config_key(P) == key
        sweep = rec["sweep"]
        assert sorted(_variant(r) for r in sweep) == sorted(_variant(c) for c in at.candidates(P)), key
        assert all(r["ms_per_rhs"] > 0 for r in sweep)
        best = min(sweep, key=lambda r: r["ms_per_rhs"])
        assert _variant(rec["choice"]) == _variant(best), key
        assert rec["points_per_rhs"] > 0


def test_recorded_choice_reads_the_record(tgh, tmp_path):
    at = tgh.autotune
    data = json.loads(RECORD.read_text())
    for key, rec in data.items():
        assert at.recorded_choice(_fake_problem(key), path=RECORD) == rec["choice"]
    # a TMA choice recorded for a configuration the TMA kernel does not cover is not applied
    bad = tmp_path / "t.json"
    bad.write_text(json.dumps({"q4_n8_fp64_interior": {"choice": {"pi": "tma", "threads": 128, "pi_mb": 4},
                                                       "sweep": [], "points_per_rhs": 1}}))
    assert at.recorded_choice(_fake_problem("q4_n8_fp64_interior"), path=bad) is None
    # an unknown configuration has no record
    assert at.recorded_choice(_fake_problem("q6_n16_fp64_nointerior"), path=RECORD) is None
