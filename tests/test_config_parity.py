"""Parity of the CUDA slice loop with the CPU oracle on the benchmark workloads themselves.

The golden-deck tests pin the arithmetic on the reference's own regression inputs; these run the
workloads the benchmark times, at their full sizes, against the oracle on the same seeded inputs:

* linear_wake_64 (64 x 64 x 100, predictor-corrector Bx/By, 1e5-particle driver): every step
  0 .. 10 (Hipace.cpp:393-554), all predictor-corrector field components after each step, and the
  beam after the last one;
* blowout_255 (255 x 255 x 256, explicit solver with multigrid at the production tolerance 1e-4,
  1e6-particle driver): one whole step (Hipace.cpp:556-728 for every slice), field components
  over all slices, the pushed beam and the plasma;
* channel_1023 (1023 x 1023 x 1024, 4.2M plasma particles in a parabolic channel, 4e6-particle
  driver): the first 64 slices of step 0 through the per-slice surface (hpq_begin_step +
  hpq_solve_slice), fields compared on the slices where the driver is present.

Bar: relative L2 <= 1e-10 per component. Both sides draw the driver from the deck's seed (the
library in hpq_init, the oracle on its own); the first test checks that the draws are identical.
"""
import numpy as np
import pytest

import hipace2_b200 as hp
from cases import config
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-10
BEAM_KEYS = ("x", "y", "z", "w", "ux", "uy", "uz")


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d


def by_id(beam):
    order = np.argsort(beam["id"], kind="stable")
    return {k: v[order] for k, v in beam.items()}


def pair(name, graphs=True):
    text = config(name)
    g = hp.Hipace(text, graphs=graphs)
    g.init_data()
    o = Oracle(text)
    o.init_beams()
    return g, o


@pytest.mark.parametrize("name", ["linear_wake_64", "blowout_255"])
def test_oracle_draws_the_library_beam(name):
    g, o = pair(name)
    bg, bo = by_id(g.get_beam(0)), by_id(o.get_beam(0))
    assert np.array_equal(bg["id"], bo["id"])
    for k in BEAM_KEYS:
        assert np.array_equal(bg[k], bo[k]), k
    g.close()


PC_COMPS = ["Psi", "Ez", "ExmBy", "EypBx", "Bx", "By", "Bz", "jx", "jy", "jz", "rhomjz"]


def test_linear_wake_64_every_step_matches_oracle():
    g, o = pair("linear_wake_64")
    g.set_diag(PC_COMPS)
    o.set_diag(PC_COMPS)
    for s in range(11):
        g.step(s)
        assert o.step(s) == 0
        for k in PC_COMPS:
            e = rel_l2(g.get_diag(k), o.get_diag(k))
            assert e <= TOL, (s, k, e)
    bg, bo = by_id(g.get_beam(0)), by_id(o.get_beam(0))
    assert np.array_equal(bg["id"], bo["id"])
    for k in BEAM_KEYS:
        e = rel_l2(bg[k], bo[k])
        assert e <= TOL, (k, e)
    g.close()


EXPLICIT_COMPS = ["Psi", "Ez", "ExmBy", "EypBx", "Bx", "By", "Bz", "jz_beam", "rhomjz", "chi", "Sx", "Sy"]


def test_blowout_255_whole_step_matches_oracle():
    g, o = pair("blowout_255")
    g.set_diag(EXPLICIT_COMPS)
    o.set_diag(EXPLICIT_COMPS)
    g.step(0)
    assert o.step(0) == 0
    for k in EXPLICIT_COMPS:
        e = rel_l2(g.get_diag(k), o.get_diag(k))
        assert e <= TOL, (k, e)
    bg, bo = by_id(g.get_beam(0)), by_id(o.get_beam(0))
    assert np.array_equal(bg["id"], bo["id"])
    for k in BEAM_KEYS:
        e = rel_l2(bg[k], bo[k])
        assert e <= TOL, (k, e)
    pg, po = g.get_plasma(0), o.get_plasma(0)
    assert np.array_equal(pg["valid"], po["valid"])
    v = po["valid"] > 0
    for k in ("x", "y", "ux", "uy", "psi"):
        e = rel_l2(pg[k][v], po[k][v])
        assert e <= TOL, (k, e)
    g.close()


def test_channel_1023_head_slices_match_oracle():
    g, o = pair("channel_1023")
    nz = g.n_cell[2]
    # rhomjz is left out here: ahead of the wake the electrons' charge cancels the ion background
    # to ~1e-6, so its relative error measures that cancellation (it is compared over a whole
    # step in the blowout test); Psi, solved from it, is compared
    comps = ["Psi", "Ez", "ExmBy", "Bx", "By", "jz_beam", "chi"]
    g.begin_step(0)
    o.begin_step(0)
    checked = 0
    for s in range(nz - 1, nz - 65, -1):
        g.solve_one_slice(s)
        assert o.solve_slice(s, 0) == 0
        if s % 16 == 0:
            ref_jz = o.get_field("jz_beam")
            if not np.any(ref_jz):
                continue  # ahead of the driver the fields are rounding noise on both sides
            for k in comps:
                e = rel_l2(g.get_field(k), o.get_field(k))
                assert e <= TOL, (s, k, e)
            checked += 1
    assert checked >= 3
    g.end_step()
    g.close()
