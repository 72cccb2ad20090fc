"""qsfb-distfind (the reference's distfind command line over libqsfb200.so) on the GPU:
its outputs equal the API's on the same codes, in every mode."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def cli(args, stdin=""):
    exe = ROOT / "qubitserf_b200" / "qsfb-distfind"
    p = subprocess.run([str(exe), *args], input=stdin, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr
    return p.stdout.strip()


def paulis(Hx, Hz):
    rows = ["".join("X" if b else "I" for b in r) for r in Hx]
    rows += ["".join("Z" if b else "I" for b in r) for r in Hz]
    return "\n".join(rows) + "\n"


def test_cli_modes_match_the_api(golden, tmp_path):
    Hx, Hz = golden.mats("steane")
    text = paulis(Hx, Hz)
    assert cli([], text) == "3"
    assert cli(["--zx"], text) == "3 3"
    assert cli(["--z"], text) == "3"
    assert cli(["--mitm", "--x"], text) == "3"
    assert cli(["--gpu", "--mitm", "--zx"], text) == "3 3"
    # blank line ends the input, '.' and '_' are identity
    assert cli([], text.replace("I", ".") + "\nXXXXXXX\n") == "3"
    Hx, Hz = golden.mats("toric4")
    hx, hz = tmp_path / "hx.txt", tmp_path / "hz.txt"
    hx.write_text("\n".join(" ".join(str(int(b)) for b in r) for r in Hx) + "\n")
    hz.write_text("\n\n".join(" ".join(str(int(b)) for b in r) for r in Hz) + "\n")
    assert cli(["--hx", str(hx), "--hz", str(hz)]) == "4"
    assert cli(["--hx", str(hx), "--hz", str(hz), "--zx", "--mitm"]) == "4 4"
    gx, gz = golden.mats("bacon_shor3")
    assert cli(["--subsystem"], paulis(gx, gz)) == str(golden.results["bacon_shor3"]["distance"])


def test_cli_operator_weight(golden, native):
    res = golden.results["opw_1"]
    Gx, Gz, z, x = golden.mats("opw_1")
    n = Gx.shape[1]
    op = "".join("Y" if (z[j] and x[j]) else "Z" if z[j] else "X" if x[j] else "I"
                 for j in range(n))
    gens = paulis(Gx, Gz)
    assert cli(["-o", op, "--zx"], gens) == f"{res['z_weight']} {res['x_weight']}"
    assert cli(["--operator", op], gens) == str(max(res["z_weight"], res["x_weight"]))
    assert cli(["-o", op, "--zx", "--mitm"], gens) == f"{res['z_weight']} {res['x_weight']}"
