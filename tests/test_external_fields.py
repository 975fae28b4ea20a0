"""External beam fields (<beam>.external_E/B(x,y,z,t), BeamParticleContainer.cpp:72-86, applied in
the beam push, BeamParticleAdvance.cpp:99, 197; ExternalFields.H:29-56) on the GPU.

* beam_evolution.1Rank: the reference's regression test of a beam focused by an external linear
  E field over 20 steps; the library's beam entering step 20 and the fields of step 20 must
  match the oracle to 1e-10 and the reference's checksums to its CUDA tolerance 1e-7;
* a deck with time-dependent external E and B (the time argument is the step's start time),
  against the oracle over three steps.
"""
import numpy as np
import pytest

import hipace2_b200 as hp
from cases import EXPLICIT_MOVING, GOLDEN
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d


def by_id(beam):
    o = np.argsort(beam["id"], kind="stable")
    return {k: v[o] for k, v in beam.items()}


def test_beam_evolution_golden_on_gpu():
    case = GOLDEN["beam_evolution.1Rank"]
    text = case["input"]
    comps = sorted(case["fields"])
    g = hp.Hipace(text, graphs=True)
    g.init_data()
    o = Oracle(text)
    o.init_beams()
    g.set_diag(comps)
    o.set_diag(comps)
    n = case["beam_after_steps"]
    for s in range(n):
        g.step(s)
        assert o.step(s) == 0
    bg, bo = by_id(g.get_beam(0)), by_id(o.get_beam(0))
    gold = case["beam"]
    for k in ("x", "y", "z", "ux", "uy", "uz", "w"):
        assert rel_l2(bg[k], bo[k]) <= 1e-10, k
        assert np.abs(bg[k]).sum() == pytest.approx(gold[k], rel=1e-7, abs=1e-300), k
    g.step(n)
    assert o.step(n) == 0
    for k in comps:
        a, b = g.get_diag(k), o.get_diag(k)
        assert rel_l2(a, b) <= 1e-10, (k, rel_l2(a, b))
        assert np.abs(a).sum() == pytest.approx(case["fields"][k], rel=1e-7, abs=1e-300), k
    g.close()


TIMED = EXPLICIT_MOVING.replace("beam.density = 5.", "beam.density = 0.5") + (
    "beam.external_E(x,y,z,t) = \"0.2*x*(1+0.01*t)\" \"0.2*y\" \"0.001*z\"\n"
    "beam.external_B(x,y,z,t) = \"0.05*y\" \"-0.05*x*cos(0.02*t)\" \"0.01\"\n")


def test_time_dependent_external_fields_match_oracle():
    g = hp.Hipace(TIMED, graphs=True)
    g.init_data()
    o = Oracle(TIMED)
    o.set_beam(0, g.get_beam(0))
    comps = ["Ez", "Bx", "By", "jz_beam"]
    g.set_diag(comps)
    o.set_diag(comps)
    for s in range(3):
        g.step(s)
        assert o.step(s) == 0
    bg, bo = by_id(g.get_beam(0)), by_id(o.get_beam(0))
    assert np.array_equal(bg["id"], bo["id"])
    for k in ("x", "y", "z", "ux", "uy", "uz", "w"):
        assert rel_l2(bg[k], bo[k]) <= 1e-10, k
    for k in comps:
        assert rel_l2(g.get_diag(k), o.get_diag(k)) <= 1e-10, k
    g.close()
