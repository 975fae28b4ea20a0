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
