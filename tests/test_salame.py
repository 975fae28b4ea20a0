"""SALAME beam loading (src/salame/Salame.cpp): in step 0 the witness weights are rescaled slice
by slice so that the witness-current-weighted Ez of the next slice equals the target.

The reference has no SALAME regression golden; the oracle's restatement is checked by the
property the algorithm is built for (the flattened Ez, exact up to the solver tolerance when the
plasma response is pushed, `salame_do_advance = 1`), and the GPU path against the oracle."""
import numpy as np
import pytest

import hipace2_b200 as hp
from oracle_lib import Oracle

DECK = """
amr.n_cell = 33 33 40
hipace.normalized_units = 1
max_step = 1
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -6. -6. -8.
geometry.prob_hi =  6.  6.  4.
beams.names = driver witness
driver.injection_type = fixed_weight
driver.num_particles = 20000
driver.position_mean = 0. 0. 1.5
driver.position_std = 0.4 0.4 0.6
driver.density = 4.
driver.u_mean = 0. 0. 2000.
driver.u_std = 0. 0. 0.
witness.injection_type = fixed_weight
witness.profile = can
witness.zmin = -6.5
witness.zmax = -5.0
witness.num_particles = 10000
witness.position_mean = 0. 0. 0.
witness.position_std = 0.2 0.2 1.
witness.density = 1.
witness.u_mean = 0. 0. 2000.
witness.u_std = 0. 0. 0.
witness.do_salame = 1
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
hipace.MG_tolerance_rel = 1e-12
"""
FIRST = 9  # head slice of the witness in DECK (z in [-5.3, -5.0))


def beams(seed=1, n_drv=20000, n_wit=10000, wit=(-6.5, -5.0)):
    rng = np.random.default_rng(seed)
    drv = {"x": rng.normal(0, 0.4, n_drv), "y": rng.normal(0, 0.4, n_drv), "z": rng.normal(1.5, 0.6, n_drv),
           "w": np.full(n_drv, 4e-3), "ux": np.zeros(n_drv), "uy": np.zeros(n_drv), "uz": np.full(n_drv, 2000.),
           "id": np.arange(1, n_drv + 1, dtype=np.int64)}
    w = {"x": rng.normal(0, 0.2, n_wit), "y": rng.normal(0, 0.2, n_wit), "z": rng.uniform(wit[0], wit[1], n_wit),
         "w": np.full(n_wit, 5e-4), "ux": np.zeros(n_wit), "uy": np.zeros(n_wit), "uz": np.full(n_wit, 2000.),
         "id": np.arange(1, n_wit + 1, dtype=np.int64)}
    return drv, w


def run_oracle(text, steps=1, wit=(-6.5, -5.0)):
    o = Oracle(text)
    d, w = beams(wit=wit)
    o.set_beam(0, d)
    o.set_beam(1, w)
    o.set_diag(["Ez", "jz_beam", "Bx", "By"])
    for s in range(steps):
        assert o.step(s) == 0
    return o


def flatness(Ez, jz, first):
    """Relative deviation of sum(jz(s) Ez(s-1)) / sum(jz(s)) from the target sum(jz(s) Ez_first)
    / sum(jz(s)) for every witness slice s."""
    out = []
    for s in range(first, 0, -1):
        if jz[s].sum() == 0:
            continue
        t = (jz[s] * Ez[first]).sum() / jz[s].sum()
        a = (jz[s] * Ez[s - 1]).sum() / jz[s].sum()
        out.append(abs(a - t) / abs(t))
    return np.array(out)


@pytest.mark.parametrize("advance,bound", [("1", 1e-6), ("0", 3e-4)])
def test_oracle_flattens_ez(advance, bound):
    o = run_oracle(DECK + "\nhipace.salame_do_advance = %s\n" % advance)
    log = o.salame_log()
    assert set(log[:, 0].astype(int)) == {9, 8, 7, 6, 5}
    # converged (|W - 1| below the tolerance) or at the iteration limit
    last = {int(s): W for s, _, W in log}
    assert all(abs(W - 1) < 5e-3 for W in last.values()), last
    dev = flatness(o.get_diag("Ez"), o.get_diag("jz_beam"), FIRST)
    assert len(dev) == 5 and dev.max() < bound, dev
    # the driver is untouched; the witness weights follow the product of the slice's factors
    w = o.get_beam(1)
    assert np.all(w["w"] > 5e-4)


def test_oracle_without_salame_is_not_flat():
    o = run_oracle(DECK.replace("witness.do_salame = 1", "witness.do_salame = 0"))
    assert o.salame_log().size == 0
    dev = flatness(o.get_diag("Ez"), o.get_diag("jz_beam"), FIRST)
    assert dev.max() > 1e-2, dev


def test_oracle_overloaded_witness_is_removed():
    """A target the witness cannot reach (W < 0): its weight goes to zero from there on, and the
    particles of those slices are invalidated (Salame.cpp:139-145, 425-429)."""
    o = run_oracle(DECK.replace("witness.zmin = -6.5", "witness.zmin = -4.5")
                   .replace("witness.zmax = -5.0", "witness.zmax = -2.5"), wit=(-4.5, -2.5))
    log = o.salame_log()
    assert (log[:, 2] == 0).any()
    first_zero = int(log[log[:, 2] == 0][0, 0])
    assert all(W == 0 for s, _, W in log if s <= first_zero)
    b = o.get_beam(1)
    slices = np.floor((b["z"] + 8.0) / 0.3).astype(int)
    assert np.all(b["w"][slices < first_zero] == 0)  # invalid particles are reported with weight 0


def test_salame_input_checks():
    with pytest.raises(hp.HpqError, match="predictor-corrector"):
        hp.Hipace(DECK + "\nhipace.bxby_solver = predictor-corrector\n")
    with pytest.raises(hp.HpqError, match="zmin"):
        hp.Hipace(DECK.replace("witness.profile = can", "witness.profile = gaussian")
                  .replace("witness.zmin = -6.5\n", "").replace("witness.zmax = -5.0\n", ""))


def gpu_vs_oracle(text, precision=hp.PLAIN_FP64):
    o = run_oracle(text, steps=2)
    g = hp.Hipace(text, precision=precision, graphs=True)
    g.init_data()
    d, w = beams()
    g.set_beam(0, d)
    g.set_beam(1, w)
    g.set_diag(["Ez", "jz_beam", "Bx", "By"])
    g.step(0)
    return o, g


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("grid", ["33 33", "63 63"])
@pytest.mark.parametrize("advance", ["1", "0"])
def test_gpu_matches_oracle(grid, advance):
    text = DECK.replace("amr.n_cell = 33 33 40", "amr.n_cell = %s 40" % grid) + \
        "\nhipace.salame_do_advance = %s\n" % advance
    o = Oracle(text)
    d, w = beams()
    o.set_beam(0, d)
    o.set_beam(1, w)
    o.set_diag(["Ez", "jz_beam", "Bx", "By"])
    assert o.step(0) == 0
    g = hp.Hipace(text, graphs=True)
    g.init_data()
    g.set_beam(0, d)
    g.set_beam(1, w)
    g.set_diag(["Ez", "jz_beam", "Bx", "By"])
    g.step(0)
    lo, lg = o.salame_log(), g.salame_log()
    assert lo.shape == lg.shape, (lo.shape, lg.shape)
    np.testing.assert_array_equal(lo[:, :2], lg[:, :2])
    assert np.abs(lo[:, 2] - lg[:, 2]).max() <= 1e-9 * np.abs(lo[:, 2]).max()
    for k in ("Ez", "jz_beam", "Bx", "By"):
        e = rel_l2(g.get_diag(k), o.get_diag(k))
        assert e <= 1e-10, (k, e)
    ob, gb = o.get_beam(1), g.get_beam(1)
    oo, go = np.argsort(ob["id"]), np.argsort(gb["id"])
    for k in ("w", "x", "uz"):
        assert np.abs(ob[k][oo] - gb[k][go]).max() <= 1e-10 * np.abs(ob[k]).max(), k
    # the next step runs without SALAME (graph replay) and still matches
    assert o.step(1) == 0
    g.step(1)
    assert g.salame_log().shape == lg.shape
    for k in ("Ez", "Bx"):
        e = rel_l2(g.get_diag(k), o.get_diag(k))
        assert e <= 1e-10, (k, e)


@pytest.mark.gpu
def test_gpu_mixed_precision_flattens():
    g = hp.Hipace(DECK, precision=hp.MIXED, graphs=True)
    g.init_data()
    d, w = beams()
    g.set_beam(0, d)
    g.set_beam(1, w)
    g.set_diag(["Ez", "jz_beam"])
    g.step(0)
    dev = flatness(g.get_diag("Ez"), g.get_diag("jz_beam"), FIRST)
    assert len(dev) == 5 and dev.max() < 1e-4, dev


def test_oracle_salame_witness_minimises_the_adjoint_objective():
    """SALAME's flattened witness, evaluated by the adjoint's objective J (current-weighted
    variance of Ez over the witness) on the same beams: J falls by orders of magnitude from the
    injected witness, and a descent step along the adjoint gradient lowers J as well."""
    from cases import ADJOINT_SMALL, adjoint_beams
    drv, wit = adjoint_beams()
    o = Oracle(ADJOINT_SMALL)
    o.set_beam(0, drv)
    o.set_beam(1, wit)
    n = o.L.oracle_adjoint_nparams(o.h)
    ones = np.ones(n)
    J0, g = o.adjoint(ones)
    text = "\n".join(l for l in ADJOINT_SMALL.splitlines() if not l.strip().startswith("adjoint."))
    s = Oracle(text + "\nwitness.do_salame = 1\n")
    s.set_beam(0, drv)
    s.set_beam(1, wit)
    assert s.step(0) == 0
    ws = s.get_beam(1)
    w_sal = dict(zip(ws["id"].tolist(), ws["w"].tolist()))
    wit_s = dict(wit)
    wit_s["w"] = np.array([w_sal.get(i, 0.0) for i in wit["id"].tolist()])
    o2 = Oracle(ADJOINT_SMALL)
    o2.set_beam(0, drv)
    o2.set_beam(1, wit_s)
    J_sal = o2.adjoint(ones, grad=False)
    assert J_sal < 1e-4 * J0, (J_sal, J0)
    g[16:] = 0.0  # witness knots only
    step = np.maximum(ones - 0.1 / np.abs(g).max() * g, 0.0)
    assert o.adjoint(step, grad=False) < J0
