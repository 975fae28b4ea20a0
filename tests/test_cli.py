"""The command-line driver hipace2_b200/hpq (the reference's executable, src/main.cpp): input
file plus ParmParse-style overrides, error exits, and on a GPU the regression checksum of the
reference's linear-wake golden."""
import json
import os
import subprocess

import pytest

import hipace2_b200 as hp
from cases import GOLDEN, golden_input

CLI = os.path.join(os.path.dirname(hp.__file__), "hpq")


def run(args, tmp_path, text=None):
    hp.load_library()
    from hipace2_b200 import build
    build.build()
    path = tmp_path / "inputs"
    path.write_text(text if text is not None else golden_input("linear_wake.normalized.1Rank"))
    return subprocess.run([CLI, str(path)] + args, capture_output=True, text=True, timeout=600)


def test_usage(tmp_path):
    r = run(["--bogus"], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr


def test_missing_input_file(tmp_path):
    r = subprocess.run([CLI, str(tmp_path / "nope")], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot read" in r.stderr


def test_overrides_in_parmparse_forms(tmp_path):
    r = run(["--dry-run"], tmp_path)
    assert r.returncode == 0 and "n_cell 32 32 200  max_step 0" in r.stdout and "beam beam" in r.stdout
    r = run(["amr.n_cell=16", "16", "20", "max_step", "=", "3", "--dry-run"], tmp_path)
    assert r.returncode == 0 and "n_cell 16 16 20  max_step 3" in r.stdout, r.stdout + r.stderr
    r = run(["amr.n_cell=24 24 30", "--dry-run", "max_step=2"], tmp_path)
    assert r.returncode == 0 and "n_cell 24 24 30  max_step 2" in r.stdout, r.stdout + r.stderr


def test_rejected_input_exits_with_message(tmp_path):
    r = run(["lasers.names=laser", "--dry-run"], tmp_path)
    assert r.returncode == 1 and "lasers.names" in r.stderr


@pytest.mark.gpu
def test_checksum_matches_reference_golden(tmp_path):
    """hpq <linear_wake deck> --checksum against the reference's checksum JSON at its CUDA
    tolerance (1e-7)."""
    name = "linear_wake.normalized.1Rank"
    r = run(["--checksum", "--quiet"], tmp_path)
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout)
    case = GOLDEN[name]
    for k, want in case["fields"].items():
        assert got["lev=0"][k] == pytest.approx(want, rel=1e-7, abs=1e-9), (k, got["lev=0"][k], want)
    for k in ("x", "y", "z", "ux", "uy", "uz", "w"):
        assert got["beam"][k] == pytest.approx(case["beam"][k], rel=1e-7, abs=1e-9), k
    assert got["beam"]["num_particles"] == case["beam"]["charge"]
