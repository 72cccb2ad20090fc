"""The reference's own, unmodified Python package (python/qubitserf, built beside the reference
libraries under oracle/_ref) driving this library through its documented override,
QUBITSERF_LIB (python/qubitserf/_native.py:36-42, 88-96): its ctypes signatures, struct
layouts and rc -> exception mapping (python/qubitserf/distfind/_native.py:15-133) bind the
drop-in ABI, and classical_distance / css_distance / subsystem_css_distance /
stabilizer_distance / operator_weight with method="bz", backend="gpu" return the golden
values.  Runs in a child process so the override takes effect before the package loads."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_PY = ROOT / "oracle" / "_ref" / "python"

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from qubitserf import distfind as df
gold = json.load(open(sys.argv[2]))
arr = np.load(sys.argv[3])
mats = lambda name: [arr[f"{name}__{i}"] for i in range(gold[name]["nmats"])]
which = {"M": "min", "Z": "z", "X": "x"}
out = {"backends": sorted(df.available_backends()), "values": {}}
for name, r in gold.items():
    m = mats(name)
    w = which.get(r.get("which", "M"), "min")
    if r["kind"] == "classical":
        v = df.classical_distance(m[0], method="bz", backend="gpu")
    elif r["kind"] == "css":
        v = df.css_distance(m[0], m[1], method="bz", which=w, backend="gpu")
    elif r["kind"] == "subsystem":
        v = df.subsystem_css_distance(m[0], m[1], method="bz", which=w, backend="gpu")
    elif r["kind"] == "stabilizer":
        v = df.stabilizer_distance(m[0], method="bz", which=w, backend="gpu")
    elif r["kind"] == "opweight":
        v = df.operator_weight(m[0], m[1], (m[2], m[3]), method="bz", backend="gpu")
    else:
        continue
    out["values"][name] = int(v)
try:
    df.classical_distance(mats("hamming3")[0], method="bz", backend="cpu")
    out["cpu"] = "returned"
except RuntimeError as e:
    out["cpu"] = "RuntimeError"
print(json.dumps(out))
"""


def run_reference_python(extra_env=None):
    if not (REF_PY / "qubitserf" / "distfind" / "api.py").exists():
        pytest.skip("the reference Python package was not copied under oracle/_ref")
    env = dict(os.environ)
    env["QUBITSERF_LIB"] = str(ROOT / "qubitserf_b200" / "libqsfb200.so")
    env.pop("DISTFIND_LIB", None)
    env.pop("CODEAUT_LIB_PATH", None)
    env.update(extra_env or {})
    g = ROOT / "tests" / "golden"
    p = subprocess.run([sys.executable, "-c", SCRIPT, str(REF_PY), str(g / "golden.json"),
                        str(g / "golden.npz")], env=env, capture_output=True, text=True,
                       timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_reference_python_over_the_drop_in(golden):
    out = run_reference_python()
    assert "gpu" in out["backends"]
    assert out["cpu"] == "RuntimeError"   # no CPU path: rc 5 surfaces as RuntimeError
    assert len(out["values"]) >= 60
    for name, v in out["values"].items():
        r = golden.results[name]
        want = max(r["z_weight"], r["x_weight"]) if r["kind"] == "opweight" else r["distance"]
        assert v == want, (name, v, want)
