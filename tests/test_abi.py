"""The C-ABI library loads and exports every entry point of include/hpq.h (no GPU needed)."""
import ctypes
import os
import re

import pytest

import hipace2_b200 as hp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "hpq.h")).read()
    return sorted(set(re.findall(r"\b(hpq_[a-z_]+)\s*\(", text)))


def test_header_matches_binding():
    assert declared() == sorted(hp.EXPORTS)


def test_library_exports_all_symbols():
    L = hp.load_library()
    for name in declared():
        assert hasattr(L, name), name


def test_create_rejects_bad_input():
    L = hp.load_library()
    h = ctypes.c_void_p()
    rc = L.hpq_create(b"amr.n_cell = 8 8 8\n", ctypes.byref(h))
    assert rc == 1
    assert b"geometry.prob_lo" in L.hpq_create_error()


def test_create_rejects_unsupported_feature():
    from cases import golden_input
    text = golden_input("linear_wake.normalized.1Rank") + "\namr.max_level = 1\n"
    with pytest.raises(hp.HpqError) as e:
        hp.Hipace(text)
    assert "mesh refinement" in str(e.value)


def test_calls_out_of_order_are_state_errors():
    from cases import golden_input
    sim = hp.Hipace(golden_input("linear_wake.normalized.1Rank"))
    with pytest.raises(hp.HpqError) as e:
        sim.step(0)
    assert e.value.code == 3


def test_queries_without_gpu():
    """Grid, max_step, diagnostic size, beam names and time are answered from the inputs."""
    from cases import golden_input
    text = golden_input("linear_wake.normalized.1Rank") + "\nmax_step = 4\ndiagnostic.diag_type = xz\n"
    sim = hp.Hipace(text)
    L = sim.L
    assert sim.max_step == 4
    nx, ny, nz = sim.n_cell
    n = ctypes.c_int64()
    assert L.hpq_diag_count(sim.h, ctypes.byref(n)) == 0 and n.value == nz * nx
    assert L.hpq_beam_name(sim.h, 0) == b"beam" and L.hpq_beam_name(sim.h, 1) is None
    assert sim.time() == 0.0


def test_shared_prefix_keys_of_unbuilt_features_are_rejected():
    """Keys the reference also reads under beams.* / plasmas.* (queryWithParserAlt) for features
    this build does not have are errors, not silently ignored."""
    from cases import golden_input
    base = golden_input("linear_wake.normalized.1Rank")
    for extra, word in (("beams.do_radiation_reaction = 1", "radiation"),
                        ("plasmas.insitu_period = 5", "in-situ"),
                        ("plasma.do_symmetrize = 1", "symmetrized"),
                        ("plasmas.fine_ppc = 2 2", "mesh refinement"),
                        ("hipace.deposit_rho_individual = 1", "per-species")):
        with pytest.raises(hp.HpqError) as e:
            hp.Hipace(base + "\n" + extra + "\n")
        assert word in str(e.value), (extra, str(e.value))
    hp.Hipace(base + "\nplasmas.insitu_period = 0\n")  # switched off: accepted
    # orders outside 0..3 are rejected when the deck is read
    with pytest.raises(hp.HpqError) as e:
        hp.Hipace(base + "\nhipace.depos_order_xy = 4\n")
    assert "0, 1, 2 or 3" in str(e.value)
