"""The autotuner's search rule, without a GPU (its measurements are replaced by a cost
model): a candidate replaces the current value only when its win repeats beside it, a
one-off lucky measurement changes nothing, the closing comparison against the defaults
guards a whole group of knobs, and every knob the tuner writes is a key the library reads."""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

import pytest

from qubitserf_b200 import tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _args():
    return argparse.Namespace(min_gain=0.01, codes=8, steps=1, warmup=0)


def test_repeated_win_is_adopted(monkeypatch):
    # one knob value is 10% faster every time it is measured; nothing else matters
    def fake(mode, values, args):
        return 27.0 if values["tc_job_tiles.large"] == 32 else 30.0

    monkeypatch.setattr(tune, "measure", fake)
    log = []
    values, best = tune.search("resident", tune.RESIDENT_KNOBS, dict(tune.DEFAULTS), _args(), log)
    assert values["tc_job_tiles.large"] == 32 and best == pytest.approx(27.0)
    assert all(values[k] == tune.DEFAULTS[k] for k in values if k != "tc_job_tiles.large")
    assert ("resident", "tc_job_tiles.large (again, against current)", 32, 27.0) in log


def test_one_off_win_is_not_adopted(monkeypatch):
    seen = {"n": 0}

    def fake(mode, values, args):
        # the first measurement of exec_groups = 2 is lucky, every later one is slower
        if values["exec_groups"] == 2:
            seen["n"] += 1
            return 27.0 if seen["n"] == 1 else 30.5
        return 30.0

    monkeypatch.setattr(tune, "measure", fake)
    values, best = tune.search("resident", tune.RESIDENT_KNOBS, dict(tune.DEFAULTS), _args(), [])
    assert values == tune.DEFAULTS and best == pytest.approx(30.0)
    assert seen["n"] == 2   # measured once more, beside the current value, and rejected


def test_gain_below_threshold_is_ignored(monkeypatch):
    # a 0.5% win is inside the 1% noise margin
    def fake(mode, values, args):
        return 29.85 if values["batch_chunks"] == 2 else 30.0

    monkeypatch.setattr(tune, "measure", fake)
    values, _ = tune.search("e2e", tune.E2E_KNOBS, dict(tune.DEFAULTS), _args(), [])
    assert values == tune.DEFAULTS


def test_closing_comparison_restores_defaults(monkeypatch, tmp_path):
    # the sweep adopts a value whose gain does not survive the closing measurement beside
    # the defaults: the group goes back to its defaults and the table says +0.0%
    state = {"closing": False}

    def fake(mode, values, args):
        if mode == "resident" and values["exec_groups"] == 4 and not state["closing"]:
            return 27.0
        return 30.0

    real_search = tune.search

    def search_then_close(*a, **k):
        out = real_search(*a, **k)
        if a[0] == "e2e":
            state["closing"] = True
        return out

    class _Lib:
        @staticmethod
        def qsfb_device_name():
            return b"fake device"

    monkeypatch.setattr(tune, "measure", fake)
    monkeypatch.setattr(tune, "search", search_then_close)
    from qubitserf_b200 import _native
    monkeypatch.setattr(_native, "backend_available", lambda b: True)
    monkeypatch.setattr(_native, "lib", lambda: _Lib())
    out = tmp_path / "tuning.txt"
    monkeypatch.setattr(sys, "argv", ["tune", "--out", str(out)])
    tune.main()
    table = out.read_text()
    rows = dict(l.split() for l in table.splitlines() if l and not l.startswith("#"))
    assert rows["exec_groups"] == str(tune.DEFAULTS["exec_groups"])
    assert "(+0.0% certificates/s)" in table


def test_env_for_names_the_library_overrides():
    env = tune.env_for({"tc_job_tiles.large": 32, "batch_first_permille": 62})
    assert env["QSFB_TUNING"] == "/nonexistent"   # candidates start from the defaults
    assert env["QSFB_TUNE_TC_JOB_TILES_LARGE"] == "32"
    assert env["QSFB_TUNE_BATCH_FIRST_PERMILLE"] == "62"


def test_every_knob_is_a_library_key(native, tmp_path):
    # a table of every knob at its last candidate value reads back unchanged
    chosen = {k: c[-1] for k, c in tune.RESIDENT_KNOBS + tune.E2E_KNOBS}
    table = tmp_path / "t.txt"
    table.write_text("".join(f"{k} {v}\n" for k, v in chosen.items()))
    code = ("import sys, json; sys.path.insert(0, sys.argv[1]); "
            "from qubitserf_b200 import _native as N; print(json.dumps(N.tuning()))")
    p = subprocess.run([sys.executable, "-c", code, ROOT],
                       env=dict(os.environ, QSFB_TUNING=str(table)), capture_output=True,
                       text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    t = json.loads(p.stdout.strip().splitlines()[-1])
    for k, v in chosen.items():
        assert t[k] == v, k
