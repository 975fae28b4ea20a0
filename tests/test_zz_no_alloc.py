"""The allocation-free Poisson entry point against the slice loop's own Poisson solve.

hpq_poisson_dirichlet_noalloc serves callers that cannot allocate device memory while they
solve (stream capture, externally owned memory pools, real-time loops); its temporaries live in
a fixed device array inside the library. Here it is called through the C ABI, twice in a row,
on right-hand sides taken from the slice loop (the Psi source -rhomjz/epsilon0 of two slices),
and its solutions must equal the Psi computed by the regular entry points (hpq_step /
hpq_solve_slice + hpq_get_field) to the tolerance of the parity tests. This file sorts last so
that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import hipace2_b200 as hp
from cases import EXPLICIT_FFT

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_noalloc_poisson_matches_slice_solver_twice():
    import torch

    text = EXPLICIT_FFT.replace("hipace.MG_tolerance_rel = 1e-12", "hipace.MG_tolerance_rel = 1e-4")
    sim = hp.Hipace(text, graphs=False)
    sim.init_data()
    nx, ny, nz = sim.n_cell
    sim.begin_step(0)
    picks = {nz // 2 + 2: None, nz // 2 - 3: None}
    for s in range(nz - 1, -1, -1):
        sim.solve_one_slice(s)
        if s in picks:
            picks[s] = (sim.get_field("rhomjz"), sim.get_field("Psi"))
    sim.end_step()
    dx = (6.0 - (-6.0)) / nx
    L = hp.load_library()
    stream = torch.cuda.current_stream()
    for s, (rhomjz, psi) in picks.items():
        assert np.abs(psi).max() > 0
        f = torch.from_numpy(np.ascontiguousarray(-rhomjz)).cuda()   # -rhomjz / epsilon0, epsilon0 = 1
        u = torch.full_like(f, float("nan"))
        rc = L.hpq_poisson_dirichlet_noalloc(ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(u.data_ptr()),
                                             nx, ny, dx, dx, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = u.cpu().numpy()
        assert rel_l2(got, psi) <= 1e-10, (s, rel_l2(got, psi))


def test_noalloc_poisson_rejects_sizes_beyond_the_limit():
    L = hp.load_library()
    dummy = ctypes.c_void_p(16)
    assert L.hpq_poisson_dirichlet_noalloc(dummy, dummy, 2047, 2047, 0.1, 0.1, None) == 7
    assert L.hpq_poisson_dirichlet_noalloc(dummy, dummy, 100, 100, 0.1, 0.1, None) == 6


@pytest.mark.parametrize("nx,ny", [(127, 63), (127, 255), (1023, 1023)])
def test_noalloc_poisson_matches_oracle_on_rectangular_and_largest_grids(nx, ny):
    """Non-square grids (the x and y twiddle tables and transform lengths differ) and the
    largest grid the scratch array holds, against the CPU oracle's DST-I solve; two calls in a
    row with different right-hand sides, so the second one runs on the first one's leftovers."""
    import torch
    from oracle_lib import lib

    L = hp.load_library()
    O = lib()
    rng = np.random.default_rng(nx * 7 + ny)
    dx, dy = 0.05, 0.07
    stream = torch.cuda.current_stream()
    for _ in range(2):
        f = rng.standard_normal((ny, nx))
        want = np.zeros_like(f)
        assert O.oracle_poisson_dirichlet(f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          want.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          nx, ny, dx, dy) == 0
        fd = torch.from_numpy(f).cuda()
        u = torch.full_like(fd, float("nan"))
        rc = L.hpq_poisson_dirichlet_noalloc(ctypes.c_void_p(fd.data_ptr()), ctypes.c_void_p(u.data_ptr()),
                                             nx, ny, dx, dy, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = u.cpu().numpy()
        assert rel_l2(got, want) <= 1e-10, rel_l2(got, want)
