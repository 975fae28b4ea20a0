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
# deterministic cases only: the statistical ones draw their beam from a random stream
CASES = {k: v for k, v in json.load(open(os.path.join(HERE, "golden", "golden_cases.json"))).items()
         if not v.get("statistical")}


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
    """The injected beam, or the beam entering step n for cases written after n steps."""
    case = CASES[name]
    o = Oracle(case["input"])
    o.init_beams()
    for s in range(case.get("beam_after_steps", 0)):
        assert o.step(s) == 0
    b = o.get_beam(0)
    gold = case["beam"]
    # sum |q| over the particles: q = -1 in normalized units, -e in SI
    normalized = any(l.split("#")[0].replace(" ", "") == "hipace.normalized_units=1" for l in case["input"].splitlines())
    q = 1.0 if normalized else 1.602176634e-19
    assert len(b["x"]) == pytest.approx(gold["charge"] / q, rel=1e-12)
    # momenta are gamma*beta*c here; the reference's output holds gamma*beta (the same in
    # normalized units, c = 1)
    c = 1.0 if normalized else 299792458.0
    for k in ("x", "y", "z", "ux", "uy", "uz", "w"):
        got = np.abs(b[k]).sum() / (c if k.startswith("u") else 1.0)
        assert got == pytest.approx(gold[k], rel=1e-12, abs=1e-300), (k, got, gold[k])


def synthetic_beam(n=4000, seed=5):
    rng = np.random.default_rng(seed)
    return {"x": rng.normal(0, 0.5, n), "y": rng.normal(0, 0.5, n), "z": rng.normal(0, 1.0, n),
            "w": np.full(n, 0.01), "ux": rng.normal(0, 3, n), "uy": rng.normal(0, 3, n),
            "uz": 2000 + rng.normal(0, 10, n), "id": np.arange(1, n + 1, dtype=np.int64)}


def test_oracle_insitu_beam_moments_are_consistent():
    """In-situ beam reductions of the oracle (BeamParticleContainer.cpp:476-548): the per-slice
    particle counts cover the particles in the box, the totals are the sums over slices, [x] is a
    weighted mean, and a finite insitu_radius only removes particles."""
    from cases import EXPLICIT_MOVING
    text = EXPLICIT_MOVING + "\nbeams.insitu_period = 1\nfields.insitu_period = 1\n"
    beam = synthetic_beam()
    inside = ((beam["z"] >= -8.0) & (beam["z"] < 4.0)).sum()
    o = Oracle(text)
    o.set_beam(0, beam)
    assert o.step(0) == 0
    nz = o.nz
    flat = o.get_insitu("beam")
    sumw, npart = flat[:nz], flat[22 * nz:23 * nz]
    assert npart.sum() == pytest.approx(flat[23 * nz + 22])
    # every particle is counted in its slice; a particle that slips into the next slice during
    # the push is counted there again (the reference's "This" beam slice includes it)
    assert inside <= npart.sum() <= inside * 1.01
    assert flat[23 * nz] == pytest.approx(sumw.sum(), rel=1e-12)
    xm = flat[nz:2 * nz]
    assert np.all(np.abs(xm[npart > 0]) < 6.0)
    fields = o.get_insitu("fields")
    assert fields.size == 11 * nz and np.all(fields[2 * nz:3 * nz] >= 0)  # [Ez^2]
    o2 = Oracle(text.replace("beams.insitu_period = 1", "beams.insitu_period = 1\nbeams.insitu_radius = 0.5"))
    o2.set_beam(0, beam)
    assert o2.step(0) == 0
    assert o2.get_insitu("beam")[23 * nz + 22] < inside
