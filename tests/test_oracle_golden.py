"""Pin the CPU oracle against the reference's own regression goldens.

Each case runs the reference's example deck with the overrides of its test script and compares
sum(|Q|) over the 3-D field output of the last iteration with the reference's checksum JSON
(tests/checksum/benchmarks_json/*.json) at the reference's CPU tolerance.
"""
import json
import os

import numpy as np
import pytest

from oracle_lib import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = json.load(open(os.path.join(HERE, "golden", "golden_cases.json")))


def _max_step(text):
    m = 0
    for line in text.splitlines():
        line = line.split("#")[0]
        if "=" in line and line.split("=")[0].strip() == "max_step":
            m = int(line.split("=")[1])
    return m


@pytest.mark.parametrize("name", sorted(CASES))
def test_field_checksums(name):
    case = CASES[name]
    o = Oracle(case["input"])
    o.init_beams()
    comps = sorted(case["fields"])
    o.set_diag(comps)
    for s in range(_max_step(case["input"]) + 1):
        assert o.step(s) == 0
    rtol = max(case["rtol_cpu"], 1e-12)
    for k in comps:
        got = np.abs(o.get_diag(k)).sum()
        want = case["fields"][k]
        assert got == pytest.approx(want, rel=rtol, abs=1e-300), (k, got, want)


@pytest.mark.parametrize("name", sorted(CASES))
def test_beam_checksums(name):
    case = CASES[name]
    o = Oracle(case["input"])
    o.init_beams()
    b = o.get_beam(0)
    gold = case["beam"]
    assert len(b["x"]) == gold["charge"]          # sum |q| with q = -1 per particle
    for k in ("x", "y", "z", "ux", "uy", "uz", "w"):
        assert np.abs(b[k]).sum() == pytest.approx(gold[k], rel=1e-12, abs=1e-12), k
