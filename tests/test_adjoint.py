"""Adjoint of one step (hpq_adjoint_grad) against central finite differences of the FP64 forward,
and the GPU adjoint against the oracle's restatement of the same reverse sweep.

The reference has no adjoint; its oracle is the finite-difference derivative of the plain FP64
path. Bar: relative agreement <= 1e-4 with central differences (per parameter, relative to the
largest gradient entry), GPU vs oracle adjoint <= 1e-7.
"""
import numpy as np
import pytest

from cases import ADJOINT_SMALL, adjoint_beams, adjoint_knots
from oracle_lib import Oracle

FD_TOL = 1e-4
FD_KNOTS = (0, 3, 6, 9, 12, 15, 17, 18)


def central_difference(f, theta, k, rel=1e-4):
    h = rel * max(abs(theta[k]), 1e-3)
    tp, tm = theta.copy(), theta.copy()
    tp[k] += h
    tm[k] -= h
    return (f(tp) - f(tm)) / (2 * h)


def oracle_with_beams(text=ADJOINT_SMALL):
    o = Oracle(text)
    d, w = adjoint_beams()
    o.set_beam(0, d)
    o.set_beam(1, w)
    return o


def test_oracle_adjoint_matches_finite_differences():
    o = oracle_with_beams()
    theta = adjoint_knots()
    J, g = o.adjoint(theta)
    assert np.isfinite(J) and J > 0
    assert o.adjoint(theta, grad=False) == pytest.approx(J, rel=1e-14)
    scale = np.abs(g).max()
    for k in FD_KNOTS:
        fd = central_difference(lambda t: o.adjoint(t, grad=False), theta, k)
        assert abs(g[k] - fd) <= FD_TOL * scale, (k, g[k], fd)
    # the density knots that do not bracket z = c t = 0 have no influence
    assert g[16] == 0.0 and g[19] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("interval", [64, 16, 5])
def test_gpu_adjoint_matches_oracle_and_finite_differences(interval):
    import hipace2_b200 as hp
    text = ADJOINT_SMALL.replace("adjoint.checkpoint_interval = 16", "adjoint.checkpoint_interval = %d" % interval)
    sim = hp.Hipace(text)
    sim.init_data()
    d, w = adjoint_beams()
    sim.set_beam(0, d)
    sim.set_beam(1, w)
    theta = adjoint_knots()
    J, g = sim.adjoint(theta)
    o = oracle_with_beams(text)
    Jo, go = o.adjoint(theta)
    assert J == pytest.approx(Jo, rel=1e-9)
    scale = np.abs(go).max()
    assert np.abs(g - go).max() <= 1e-7 * scale, np.abs(g - go).max() / scale
    # the forward alone gives the same objective and leaves the state reusable
    assert sim.adjoint(theta, grad=False) == pytest.approx(J, rel=1e-12)
    if interval == 16:
        for k in FD_KNOTS:
            fd = central_difference(lambda t: sim.adjoint(t, grad=False), theta, k)
            assert abs(g[k] - fd) <= FD_TOL * scale, (k, g[k], fd)
    sim.close()


@pytest.mark.gpu
def test_reverse_mode_push_adjoint_equals_forward_mode(tmp_path):
    """The push adjoint in reverse mode (one thread per particle, the default) and in forward
    mode (HPQ_ADJ_PUSH=tangent: one thread per particle and seed) compute the same products of
    the same derivatives in another order: the gradients agree to rounding."""
    import os
    import subprocess
    import sys
    code = (
        "import sys, numpy as np; sys.path.insert(0, 'tests'); import hipace2_b200 as hp;"
        "from cases import ADJOINT_SMALL, adjoint_beams, adjoint_knots;"
        "s = hp.Hipace(ADJOINT_SMALL); s.init_data(); d, w = adjoint_beams(); s.set_beam(0, d); s.set_beam(1, w);"
        "J, g = s.adjoint(adjoint_knots()); np.save(sys.argv[1], np.concatenate([[J], g]))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for mode in ("reverse", "tangent"):
        env = dict(os.environ)
        env.pop("HPQ_ADJ_PUSH", None)
        if mode == "tangent":
            env["HPQ_ADJ_PUSH"] = "tangent"
        path = str(tmp_path / ("adj_%s.npy" % mode))
        subprocess.run([sys.executable, "-c", code, path], cwd=root, env=env, check=True, timeout=600)
        out[mode] = np.load(path)
    a, b = out["reverse"], out["tangent"]
    assert a[0] == pytest.approx(b[0], rel=1e-13)
    scale = np.abs(b[1:]).max()
    assert np.abs(a[1:] - b[1:]).max() <= 1e-10 * scale, np.abs(a[1:] - b[1:]).max() / scale


@pytest.mark.gpu
def test_adjoint_through_torch_autograd_and_step_after():
    """A thin torch.autograd.Function over hpq_adjoint_grad (harness only): backward returns the
    adjoint gradient; a normal step runs after the adjoint calls."""
    import torch
    import hipace2_b200 as hp

    sim = hp.Hipace(ADJOINT_SMALL)
    sim.init_data()
    d, w = adjoint_beams()
    sim.set_beam(0, d)
    sim.set_beam(1, w)

    class Objective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, knots):
            J, g = sim.adjoint(knots.detach().cpu().numpy().astype(np.float64))
            ctx.save_for_backward(torch.from_numpy(g))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return gJ * g

    theta = torch.tensor(adjoint_knots(), dtype=torch.float64, requires_grad=True)
    J = Objective.apply(theta)
    J.backward()
    J2, g2 = sim.adjoint(theta.detach().numpy())
    assert float(J) == pytest.approx(J2, rel=1e-12)
    assert np.allclose(theta.grad.numpy(), g2, rtol=1e-9, atol=0)
    sim.step(0)
    assert np.isfinite(sim.get_beam(1)["x"]).all()
    sim.close()


def test_oracle_adjoint_node_centred_grid():
    """Odd grid: node-centred multigrid levels, whose operator is symmetric (W = 1); density knots
    bracketing z = c t through the plasma and ion weights."""
    text = ADJOINT_SMALL.replace("amr.n_cell = 32 32 64", "amr.n_cell = 33 33 48")
    o = oracle_with_beams(text)
    theta = adjoint_knots()
    J, g = o.adjoint(theta)
    scale = np.abs(g).max()
    for k in (5, 10, 17, 18):
        fd = central_difference(lambda t: o.adjoint(t, grad=False), theta, k)
        assert abs(g[k] - fd) <= FD_TOL * scale, (k, g[k], fd)


@pytest.mark.gpu
def test_single_precision_forward_adjoint_against_fp64():
    """hpq_adjoint_grad in mixed precision: FP32 forward (and segment recomputation) recorded in
    double, FP64 reverse sweep. Against the FP64 oracle's gradient and central differences of
    the FP64 forward; the difference is the FP32 rounding of the recorded trajectory (measured
    on a B200: objective 2.0e-5, gradient 3.6e-5 of its largest entry)."""
    import hipace2_b200 as hp
    sim = hp.Hipace(ADJOINT_SMALL, precision=hp.MIXED)
    sim.init_data()
    d, w = adjoint_beams()
    sim.set_beam(0, d)
    sim.set_beam(1, w)
    theta = adjoint_knots()
    J, g = sim.adjoint(theta)
    o = oracle_with_beams()
    Jo, go = o.adjoint(theta)
    scale = np.abs(go).max()
    err = np.abs(g - go).max() / scale
    print("mixed adjoint: J rel", abs(J - Jo) / abs(Jo), "grad max diff / max", err)
    assert J == pytest.approx(Jo, rel=1e-4)
    assert err <= 1e-4, err
    for k in FD_KNOTS:
        fd = central_difference(lambda t: o.adjoint(t, grad=False), theta, k)
        assert abs(g[k] - fd) <= 2e-4 * scale, (k, g[k], fd)
    # the forward alone repeats the objective (up to the order of the FP32 atomic sums), and a
    # plain step still runs after the adjoint
    assert sim.adjoint(theta, grad=False) == pytest.approx(J, rel=1e-5)
    sim.step(0)
    sim.close()
