"""Known-answer tests of the oracle (CPU) for properties the checksum goldens do not pin.

* The Dirichlet Poisson solve by DST-I: sine modes are eigenfunctions of the 5-point Laplacian
  with the exact eigenvalue, the solve inverts that operator, and the transform applied twice is
  2(n+1) times the identity (no third-party code pins the DST here; the reference uses cuFFT or
  FFTW RODFT00, FFTPoissonSolverDirichletFast.cpp:196-328, WrapFFTW.cpp:120-125).
* Linear plasma response: on the axis of the linear-wake example (a wide flat-top driver of
  density 0.01 in a uniform plasma) the plasma charge density follows 1-D linear theory,
  rho(zeta) = kp * integral over zeta' > zeta of sin(kp (zeta' - zeta)) n_b(zeta') (normalized
  units), within the tolerance of the reference's own analysis of that example
  (examples/linear_wake/analysis.py: relative squared error < 0.025).
"""
import numpy as np

from cases import golden_input
from oracle_lib import Oracle, lib, _dp


def solve(f, dx, dy):
    ny, nx = f.shape
    u = np.zeros_like(f)
    assert lib().oracle_poisson_dirichlet(_dp(np.ascontiguousarray(f)), _dp(u), nx, ny, dx, dy) == 0
    return u


def laplacian(u, dx, dy):
    p = np.pad(u, 1)  # u = 0 one cell outside the grid
    return ((p[1:-1, 2:] - 2 * u + p[1:-1, :-2]) / dx**2 + (p[2:, 1:-1] - 2 * u + p[:-2, 1:-1]) / dy**2)


def test_sine_modes_are_eigenfunctions():
    nx, ny, dx, dy = 33, 20, 0.3, 0.45
    i = np.arange(1, nx + 1)[None, :]
    j = np.arange(1, ny + 1)[:, None]
    for k, l in ((1, 1), (5, 3), (33, 20), (17, 1)):
        f = np.sin(np.pi * k * i / (nx + 1)) * np.sin(np.pi * l * j / (ny + 1))
        lam = -4 * (np.sin(np.pi * k / (2 * (nx + 1)))**2 / dx**2 + np.sin(np.pi * l / (2 * (ny + 1)))**2 / dy**2)
        u = solve(f, dx, dy)
        assert np.abs(u - f / lam).max() <= 1e-12 * np.abs(f / lam).max(), (k, l)


def test_solve_inverts_the_five_point_laplacian():
    rng = np.random.default_rng(3)
    for nx, ny in ((31, 31), (64, 48), (7, 50)):
        f = rng.normal(size=(ny, nx))
        u = solve(f, 0.2, 0.1)
        assert np.abs(laplacian(u, 0.2, 0.1) - f).max() <= 1e-10 * np.abs(f).max()


def test_dst_twice_is_a_multiple_of_the_identity():
    rng = np.random.default_rng(5)
    for n in (1, 8, 31, 100):
        v = rng.normal(size=n)
        a, b = np.zeros(n), np.zeros(n)
        assert lib().oracle_dst1(_dp(v), _dp(a), n) == 0
        assert lib().oracle_dst1(_dp(a), _dp(b), n) == 0
        np.testing.assert_allclose(b, 2 * (n + 1) * v, rtol=0, atol=1e-11 * 2 * (n + 1) * np.abs(v).max())


def test_linear_wake_follows_linear_theory():
    text = golden_input("linear_wake.normalized.1Rank")
    o = Oracle(text)
    o.init_beams()
    o.set_diag(["rho"])
    assert o.step(0) == 0
    rho = o.get_diag("rho")              # nz x ny x nx
    nz, ny, nx = rho.shape
    axis = rho[:, ny // 2 - 1:ny // 2 + 1, nx // 2 - 1:nx // 2 + 1].mean(axis=(1, 2))
    zlo, zhi = -7.5, 2.0
    dz = (zhi - zlo) / nz
    zeta = zlo + (np.arange(nz) + 0.5) * dz
    nb = np.where((zeta >= -1.0) & (zeta <= 1.0), 0.01, 0.0)  # flat-top driver, density 0.01
    kp = 1.0
    theory = np.array([kp * dz * np.sum(np.sin(kp * (zeta[zeta > z] - z)) * nb[zeta > z]) for z in zeta])
    err = np.sum((axis - theory)**2) / np.sum(theory**2)
    assert err < 0.025, err


# The beam-in-vacuum example (examples/beam_in_vacuum/inputs_normalized with the overrides of
# tests/beam_in_vacuum.normalized.1Rank.sh), at the deposition order this build implements (2;
# the example runs order 0, which is rejected here)
BEAM_IN_VACUUM = """
amr.n_cell = 512 768 4
hipace.normalized_units = 1
max_step = 0
boundary.field = Dirichlet
boundary.particle = Periodic
geometry.prob_lo = -200. -200. -2.
geometry.prob_hi =  200.  200.  2.
beams.names = beam
beam.injection_type = fixed_ppc
beam.profile = flattop
beam.zmin = -10.
beam.zmax = 10.
beam.radius = 1.
beam.density = 1.0
beam.u_mean = 0. 0. 1.e3
beam.u_std = 0. 0. 0.
beam.ppc = 2 2 1
hipace.depos_order_xy = 2
hipace.MG_tolerance_rel = 1e-5
"""


def test_beam_in_vacuum_fields_follow_the_analytic_can_beam():
    """A long uniform beam of radius R = 1 in vacuum: Bx, By, Ex = ExmBy + By, Ey = EypBx - Bx on
    lines through the axis against the fields of a uniform cylinder (linear inside, 1/r outside;
    jz = rho = -1). The example's own analysis accepts 0.5-1.5 % at deposition order 0; order 2
    spreads the beam edge over more cells (R is 1.3-1.9 cells here), measured 1.3-2.8 %."""
    o = Oracle(BEAM_IN_VACUUM)
    o.init_beams()
    comps = ["Bx", "By", "ExmBy", "EypBx"]
    o.set_diag(comps)
    assert o.step(0) == 0
    d = {c: o.get_diag(c) for c in comps}
    nz, ny, nx = d["Bx"].shape
    k = nz // 2
    x = -200 + (np.arange(nx) + 0.5) * 400 / nx
    y = -200 + (np.arange(ny) + 0.5) * 400 / ny

    def cylinder(r, a):
        return np.where(np.abs(r) < 1.0, a * r / 2, a / (2 * r))

    By = d["By"][k, ny // 2, :]
    Bx = d["Bx"][k, :, nx // 2]
    cases = {"Bx": (Bx, -cylinder(y, -1.0)), "By": (By, cylinder(x, -1.0)),
             "Ex": (d["ExmBy"][k, ny // 2, :] + By, cylinder(x, -1.0)),
             "Ey": (d["EypBx"][k, :, nx // 2] - Bx, cylinder(y, -1.0))}
    for name, (sim, th) in cases.items():
        err = np.sum((sim - th)**2) / np.sum(th**2)
        assert err < 0.04, (name, err)
