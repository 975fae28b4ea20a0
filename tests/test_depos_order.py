"""Transverse shape orders 0..3 (hipace.depos_order_xy; ShapeFactors.H) and the three derivative
types of the explicit deposition (hipace.depos_derivative_type).

CPU: the restated shape factors are B-splines — they sum to one and reproduce linear functions
(the first moment about the particle vanishes for order >= 1), and every derivative form
differentiates a linear function exactly (sum of s'.i = 1 with the reference's sign convention,
ds = -s'); the stencil widths are the reference's (order + 1; order + type + 1; order + 3 for the
centred type).
GPU: the library matches the oracle to 1e-10 at every order with each derivative type, and with
the predictor-corrector solver at orders 1 and 3.
"""
import ctypes

import numpy as np
import pytest

from cases import EXPLICIT_MOVING, PC_SMALL
from oracle_lib import Oracle, lib


def shape(type_, ord_, xmid, ix):
    s, ds, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    assert lib().oracle_shape_factor(type_, ord_, xmid, ix, ctypes.byref(s), ctypes.byref(ds), ctypes.byref(c)) == 0
    return s.value, ds.value, c.value


def npoints(type_, ord_):
    return ord_ + 1 if type_ < 0 else (ord_ + 3 if type_ == 2 else ord_ + type_ + 1)


@pytest.mark.parametrize("ord_", [0, 1, 2, 3])
@pytest.mark.parametrize("type_", [-1, 0, 1, 2])
def test_shape_factors_are_partitions_of_unity_and_exact_for_linear_functions(type_, ord_):
    rng = np.random.default_rng(10 * ord_ + type_ + 5)
    for xmid in np.concatenate([rng.uniform(0.0, 50.0, 200), [3.0, 3.5, 7.25]]):
        pts = [shape(type_, ord_, xmid, ix) for ix in range(npoints(type_, ord_))]
        cells = [c for _, _, c in pts]
        assert cells == list(range(cells[0], cells[0] + len(cells)))  # contiguous stencil
        ssum = sum(s for s, _, _ in pts)
        assert ssum == pytest.approx(1.0, abs=1e-12)
        if type_ < 0 and ord_ >= 1:
            # cell centres sit at integer coordinates: the shape's first moment is the position
            assert sum(s * c for s, _, c in pts) == pytest.approx(xmid, abs=1e-10)
        if type_ >= 0 and ord_ >= 1:
            # -ds is the derivative weight: a linear field f_i = i has derivative 1
            assert sum(-ds * c for _, ds, c in pts) == pytest.approx(1.0, abs=1e-10)
            assert sum(ds for _, ds, _ in pts) == pytest.approx(0.0, abs=1e-12)


def test_oracle_orders_change_the_wake_but_keep_charge():
    """The wake of the same beam at orders 1 and 3 differs (shapes differ) by a few percent while
    the deposited beam charge sum jz_beam stays the same."""
    base = EXPLICIT_MOVING.replace("beam.density = 5.", "beam.density = 0.5").replace("max_step = 2", "max_step = 0")
    out = {}
    beam = None
    for o_ in (1, 2, 3):
        o = Oracle(base + "hipace.depos_order_xy = %d\n" % o_)
        o.init_beams()
        if beam is None:
            beam = o.get_beam(0)
        o.set_beam(0, beam)
        o.set_diag(["Ez", "jz_beam"])
        assert o.step(0) == 0
        out[o_] = (o.get_diag("Ez"), o.get_diag("jz_beam"))
    for o_ in (1, 3):
        assert out[o_][1].sum() == pytest.approx(out[2][1].sum(), rel=1e-12)
        d = np.linalg.norm(out[o_][0] - out[2][0]) / np.linalg.norm(out[2][0])
        assert 1e-4 < d < 0.3


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / n if n > 0 else np.linalg.norm(a - b)


COMPS = ["Psi", "Ez", "ExmBy", "EypBx", "Bx", "By", "Bz", "jx", "jy", "jz_beam", "rhomjz", "chi", "Sx", "Sy"]


@pytest.mark.gpu
@pytest.mark.parametrize("ord_", [0, 1, 3])
@pytest.mark.parametrize("dtype_", [0, 1, 2])
def test_orders_and_derivative_types_match_oracle(ord_, dtype_):
    import hipace2_b200 as hp
    text = (EXPLICIT_MOVING.replace("beam.density = 5.", "beam.density = 0.5")
            .replace("hipace.depos_order_xy = 2", "hipace.depos_order_xy = %d" % ord_)
            + "hipace.depos_derivative_type = %d\n" % dtype_)
    g = hp.Hipace(text, graphs=True)
    g.init_data()
    o = Oracle(text)
    o.set_beam(0, g.get_beam(0))
    g.set_diag(COMPS)
    o.set_diag(COMPS)
    for s in range(3):
        g.step(s)
        assert o.step(s) == 0
    for k in COMPS:
        e = rel_l2(g.get_diag(k), o.get_diag(k))
        assert e <= 1e-10, (k, e)
    bg, bo = g.get_beam(0), o.get_beam(0)
    ig, io = np.argsort(bg["id"]), np.argsort(bo["id"])
    for k in ("x", "y", "ux", "uy", "uz"):
        assert rel_l2(bg[k][ig], bo[k][io]) <= 1e-10, k
    pg, po = g.get_plasma(0), o.get_plasma(0)
    v = po["valid"] > 0
    assert np.array_equal(pg["valid"], po["valid"])
    for k in ("x", "y", "ux", "uy", "psi"):
        assert rel_l2(pg[k][v], po[k][v]) <= 1e-10, k
    g.close()


# Deterministic mode for the predictor-corrector case at order 3. At the head of the box the
# plasma electrons and the neutralising ion background cancel in rho - jz; with floating-point
# atomics the GPU's sum is sometimes exactly 0 and sometimes one rounding step off, depending on
# the order of the additions, which leaves Bx of the first slice at 0 or at ~1e-18. The
# predictor-corrector error Sum|B - B_iter| / Sum|B| (Fields.cpp, 0 when Sum|B| = 0) then jumps
# from 0 to a ratio of rounding residues, the mixing weights of the next slice flip, and that
# slice's Bx ends a few per cent off (4e-6 over the whole step). The oracle's sequential sums
# cancel exactly; the fixed-point sums of deterministic mode do too.
PC_DETERMINISTIC = {1: False, 3: True}


@pytest.mark.gpu
@pytest.mark.parametrize("ord_", [1, 3])
def test_predictor_corrector_orders_match_oracle(ord_):
    import hipace2_b200 as hp
    text = PC_SMALL + "hipace.depos_order_xy = %d\n" % ord_
    g = hp.Hipace(text, graphs=True)
    g.set_deterministic(PC_DETERMINISTIC[ord_])
    g.init_data()
    o = Oracle(text)
    o.set_beam(0, g.get_beam(0))
    comps = ["Psi", "Ez", "Bx", "By", "jx", "jz", "rhomjz"]
    g.set_diag(comps)
    o.set_diag(comps)
    for s in range(2):
        g.step(s)
        assert o.step(s) == 0
    for k in comps:
        e = rel_l2(g.get_diag(k), o.get_diag(k))
        assert e <= 1e-10, (k, e)
    g.close()


@pytest.mark.gpu
def test_predictor_corrector_order3_in_fresh_simulations():
    """Four fresh simulations in one process (graphs on and off), each with the beam it draws
    itself, in deterministic mode, against one oracle step: every run must match (with
    floating-point atomics a run can land on the other side of the predictor-corrector's
    0-or-ratio switch at the head of the box, see PC_DETERMINISTIC)."""
    import hipace2_b200 as hp
    text = PC_SMALL + "hipace.depos_order_xy = 3\n"
    comps = ["Psi", "Ez", "Bx", "By", "jx", "jz", "rhomjz"]
    ref = None
    for rep in range(4):
        g = hp.Hipace(text, graphs=rep % 2 == 0)
        g.set_deterministic(True)
        g.init_data()
        if ref is None:
            o = Oracle(text)
            o.set_beam(0, g.get_beam(0))
            o.set_diag(comps)
            assert o.step(0) == 0
            ref = {k: o.get_diag(k) for k in comps}
        g.set_diag(comps)
        g.step(0)
        for k in comps:
            e = rel_l2(g.get_diag(k), ref[k])
            assert e <= 1e-10, (rep, k, e)
        g.close()
