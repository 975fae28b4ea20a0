"""hipace.max_time (Hipace::Evolve, Hipace.cpp:401-435): the step that would cross max_time is
shortened to end on it, the step that starts on it runs with dt = 0, and then the step loop ends."""
import math

import numpy as np
import pytest

import hipace2_b200 as hp
from cases import EXPLICIT_MOVING
from oracle_lib import Oracle

TEXT = (EXPLICIT_MOVING.replace("amr.n_cell = 33 33 40", "amr.n_cell = 17 17 24")
        .replace("max_step = 2", "max_step = 6") + "\nhipace.max_time = 30\n")


def beam(n=3000, seed=11):
    rng = np.random.default_rng(seed)
    return {"x": rng.normal(0, 0.5, n), "y": rng.normal(0, 0.5, n), "z": rng.normal(0, 1.0, n),
            "w": np.full(n, 0.02), "ux": rng.normal(0, 3, n), "uy": rng.normal(0, 3, n),
            "uz": 2000 + rng.normal(0, 10, n), "id": np.arange(1, n + 1, dtype=np.int64)}


def by_id(b):
    o = np.argsort(b["id"])
    return {k: v[o] for k, v in b.items()}


def oracle_run():
    o = Oracle(TEXT)
    o.set_beam(0, beam())
    times, beams = [o.time()], [by_id(o.get_beam(0))]
    for s in range(3):
        assert o.step(s) == 0
        times.append(o.time())
        beams.append(by_id(o.get_beam(0)))
    return times, beams


def test_oracle_shortens_and_ends_the_step_loop():
    times, beams = oracle_run()
    assert times[:3] == [0.0, 20.0, 30.0] and math.isinf(times[3])
    # the dt = 0 step leaves the beam where it was
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        np.testing.assert_array_equal(beams[3][k], beams[2][k])
    # the shortened step is a step of dt = 10 from the same state (the plasma density does not
    # depend on z = c t here, so the step's start time does not matter)
    o = Oracle(TEXT.replace("hipace.dt = 20", "hipace.dt = 10").replace("hipace.max_time = 30", ""))
    b1 = dict(beams[1])
    o.set_beam(0, b1)
    assert o.step(0) == 0
    want = by_id(o.get_beam(0))
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        np.testing.assert_array_equal(beams[2][k], want[k])


@pytest.mark.gpu
def test_gpu_matches_oracle_and_stops():
    times, beams = oracle_run()
    g = hp.Hipace(TEXT, graphs=True)
    g.init_data()
    g.set_beam(0, beam())
    got_t = [g.time()]
    for s in range(3):
        g.step(s)
        got_t.append(g.time())
        b = by_id(g.get_beam(0))
        for k in ("x", "y", "z", "ux", "uy", "uz", "w"):
            want = beams[s + 1][k]
            assert np.abs(b[k] - want).max() <= 1e-9 * max(1.0, np.abs(want).max()), (s, k)
    assert got_t[:3] == times[:3] and math.isinf(got_t[3])
    with pytest.raises(hp.HpqError) as e:
        g.step(3)
    assert e.value.code == 3
    # evolve() leaves the loop the same way
    g2 = hp.Hipace(TEXT, graphs=False)
    g2.init_data()
    g2.set_beam(0, beam())
    g2.evolve()
    assert math.isinf(g2.time())
