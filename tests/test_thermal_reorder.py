"""Thermal plasma (<plasma>.u_std / temperature_in_ev) and plasma reordering (reorder_period).

The reference draws the thermal momenta u = u_mean + u_std N(0, 1) when it creates the plasma of
a step (PlasmaParticleContainerInit.cpp:282, ParticleUtil.H:113-124) and sorts the particles by
cell every reorder_period slices (PlasmaParticleContainer.cpp:197-208). Here both sides draw from
the same counter-based stream (rng.hpp), so the oracle and the library start every step from the
same plasma; the reorder is a stable sort by bin on both sides, so particle arrays stay
comparable index by index.
"""
import numpy as np
import pytest

from cases import EXPLICIT_MOVING
from oracle_lib import Oracle

# weak driver, warm plasma, reordered every 4 slices
THERMAL = (EXPLICIT_MOVING.replace("beam.density = 5.", "beam.density = 0.5")
           + "plasma.u_std = 0.05 0.04 0.03\nplasma.reorder_period = 4\n")
COLD = EXPLICIT_MOVING.replace("beam.density = 5.", "beam.density = 0.5")


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d


def shared_beam(text):
    """A beam both sides can load (the deck's seeded draw, taken from the oracle)."""
    o = Oracle(text)
    o.init_beams()
    return o.get_beam(0)


def test_oracle_thermal_momenta_have_the_requested_spread():
    o = Oracle(THERMAL.replace("plasma.reorder_period = 4\n", ""))
    o.init_beams()
    o.begin_step(0)
    p = o.get_plasma(0)
    n = p["ux"].size
    assert n > 1000
    # normalized units: u stored as u * c with c = 1
    for k, s in (("ux", 0.05), ("uy", 0.04)):
        assert abs(p[k].mean()) < 4 * s / np.sqrt(n)
        assert p[k].std() == pytest.approx(s, rel=0.05)
    # psi = sqrt(1 + u^2) - uz with uz ~ N(0, 0.03): mean above 1 - small
    assert np.all(p["psi"] > 0.8) and np.all(p["psi"] < 1.2)
    # a new step draws new momenta
    o.step(0)
    o.begin_step(1)
    q = o.get_plasma(0)
    assert not np.array_equal(q["ux"], p["ux"])


def test_oracle_temperature_sets_u_std():
    # 1 keV electrons: u_std = sqrt(T e / (m c^2)) = 0.04424
    o = Oracle(COLD + "plasma.temperature_in_ev = 1000.\n")
    o.init_beams()
    o.begin_step(0)
    ux = o.get_plasma(0)["ux"]
    assert ux.std() == pytest.approx(np.sqrt(1000 * 1.602176634e-19 / (9.1093837015e-31 * 299792458.0 ** 2)), rel=0.05)
    with pytest.raises(ValueError):
        Oracle(COLD + "plasma.temperature_in_ev = 1000.\nplasma.u_std = 0.1 0.1 0.1\n")


def test_oracle_reorder_changes_only_the_summation_order():
    """Reordering permutes particles; the fields change only by the order of the deposit sums."""
    beam = shared_beam(THERMAL)
    comps = ["Ez", "Psi", "Bx", "By", "jx", "rhomjz"]
    out = {}
    for period in (0, 4):
        o = Oracle(THERMAL.replace("plasma.reorder_period = 4", "plasma.reorder_period = %d" % period))
        o.set_beam(0, beam)
        o.set_diag(comps)
        o.step(0)
        o.step(1)
        out[period] = {k: o.get_diag(k) for k in comps}
        if period:
            # after the last slice (0, a multiple of 4) the particles are sorted by cell
            p = o.get_plasma(0)
            dx = 12.0 / 33
            key = (np.floor((p["y"] + 6.0) / dx).clip(0, 32) * 34 + np.floor((p["x"] + 6.0) / dx).clip(0, 32))
            # particles moved by one slice's push after the sort; most keys stay ordered
            assert np.mean(np.diff(key) >= 0) > 0.9
    for k in comps:
        assert rel_l2(out[4][k], out[0][k]) <= 1e-10, k


@pytest.mark.gpu
def test_thermal_reordered_plasma_matches_oracle():
    import hipace2_b200 as hp
    beam = shared_beam(THERMAL)
    comps = ["Psi", "Ez", "ExmBy", "EypBx", "Bx", "By", "Bz", "jx", "jy", "jz_beam", "rhomjz", "chi", "Sx", "Sy"]
    for graphs in (True, False):
        g = hp.Hipace(THERMAL, graphs=graphs)
        g.init_data()
        g.set_beam(0, beam)
        o = Oracle(THERMAL)
        o.set_beam(0, beam)
        g.set_diag(comps)
        o.set_diag(comps)
        for s in range(3):
            g.step(s)
            assert o.step(s) == 0
        for k in comps:
            e = rel_l2(g.get_diag(k), o.get_diag(k))
            assert e <= 1e-10, (graphs, k, e)
        pg, po = g.get_plasma(0), o.get_plasma(0)
        assert np.array_equal(pg["valid"], po["valid"])
        for k in ("x", "y", "ux", "uy", "psi"):
            e = rel_l2(pg[k], po[k])
            assert e <= 1e-10, (graphs, k, e)
        g.close()


@pytest.mark.gpu
def test_reordered_deterministic_runs_are_bit_identical():
    import hipace2_b200 as hp
    beam = shared_beam(THERMAL)
    res = []
    for _ in range(2):
        g = hp.Hipace(THERMAL, graphs=True)
        g.set_deterministic(True)
        g.init_data()
        g.set_beam(0, beam)
        g.set_diag(["Ez", "Bx"])
        for s in range(2):
            g.step(s)
        res.append((g.get_diag("Ez"), g.get_diag("Bx"), g.get_plasma(0)["x"]))
        g.close()
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_mixed_precision_reorder_keeps_positions():
    """Single precision stores positions as displacements from a lattice point carried by the
    particle; after a reorder the absolute positions must be those of the FP64 path to FP32
    accuracy, with and without reordering."""
    import hipace2_b200 as hp
    beam = shared_beam(THERMAL)
    xs = {}
    for period in (0, 4):
        text = THERMAL.replace("plasma.reorder_period = 4", "plasma.reorder_period = %d" % period)
        g = hp.Hipace(text, precision=hp.MIXED, graphs=True)
        g.init_data()
        g.set_beam(0, beam)
        g.step(0)
        p = g.get_plasma(0)
        xs[period] = (np.sort(p["x"]), np.sort(p["y"]))
        g.close()
    # the sorted coordinates of two nearly equal particle sets differ by at most the largest
    # displacement between them
    for a, b in zip(xs[0], xs[4]):
        assert np.max(np.abs(a - b)) < 1e-4
