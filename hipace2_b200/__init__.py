"""B200-native quasi-static slice loop (HiPACE++ slice solver) — Python host interface.

The product is the C-ABI library libhpq.so (include/hpq.h) built from hipace2_b200/csrc for
sm_100a. This module binds it with ctypes and mirrors the reference's driver surface:
`Hipace(inputs)` (src/Hipace.cpp:74-244), `init_data()` (:246-295), `evolve()` (:393-554) and
`solve_one_slice(islice, step)` (:556-728). There is no CPU fallback: loading fails loudly if
the library or a CUDA device is missing.
"""
import ctypes
import math
import os

import numpy as np

__all__ = ["Hipace", "HpqError", "load_library", "PLAIN_FP64", "MIXED"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhpq.so")
PLAIN_FP64, MIXED = 0, 1
ERRORS = {1: "input", 2: "cuda", 3: "state", 4: "not converged", 5: "diverged", 6: "argument"}

# every entry point declared in include/hpq.h
EXPORTS = ("hpq_create", "hpq_destroy", "hpq_last_error", "hpq_create_error", "hpq_set_precision",
           "hpq_init", "hpq_set_beam", "hpq_beam_count", "hpq_get_beam", "hpq_step",
           "hpq_begin_step", "hpq_solve_slice", "hpq_end_step", "hpq_get_field", "hpq_set_diag",
           "hpq_get_diag", "hpq_insitu_size", "hpq_get_insitu", "hpq_plasma_count", "hpq_get_plasma", "hpq_set_graphs",
           "hpq_set_deterministic", "hpq_synchronize", "hpq_stream", "hpq_get_counters", "hpq_set_profiling",
           "hpq_get_profile", "hpq_poisson_dirichlet_noalloc", "hpq_adjoint_nparams", "hpq_adjoint_grad", "hpq_n_cell",
           "hpq_max_step", "hpq_time", "hpq_diag_count", "hpq_beam_name", "hpq_salame_log",
           "hpq_beam_slice_count", "hpq_get_beam_slice", "hpq_put_beam_slice", "hpq_set_time")

_lib = None


class HpqError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hpq error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def load_library(path=None):
    """Load libhpq.so (building it first when the sources are newer and nvcc is present)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(path)
    vp, cp, i32, i64 = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int64
    dp, lp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)
    sig = {
        "hpq_create": ([cp, ctypes.POINTER(vp)], i32),
        "hpq_destroy": ([vp], None),
        "hpq_last_error": ([vp], cp),
        "hpq_create_error": ([], cp),
        "hpq_set_precision": ([vp, i32], i32),
        "hpq_init": ([vp], i32),
        "hpq_set_beam": ([vp, i32] + [dp] * 7 + [lp, i64], i32),
        "hpq_beam_count": ([vp, i32, lp], i32),
        "hpq_get_beam": ([vp, i32] + [dp] * 7 + [lp], i32),
        "hpq_step": ([vp, i32], i32),
        "hpq_begin_step": ([vp, i32], i32),
        "hpq_solve_slice": ([vp, i32], i32),
        "hpq_end_step": ([vp], i32),
        "hpq_get_field": ([vp, cp, dp], i32),
        "hpq_set_diag": ([vp, cp], i32),
        "hpq_get_diag": ([vp, cp, dp], i32),
        "hpq_plasma_count": ([vp, i32, lp], i32),
        "hpq_get_plasma": ([vp, i32, dp], i32),
        "hpq_set_graphs": ([vp, i32], i32),
        "hpq_set_deterministic": ([vp, i32], i32),
        "hpq_insitu_size": ([vp, cp, ctypes.POINTER(ctypes.c_int64)], i32),
        "hpq_get_insitu": ([vp, cp, dp], i32),
        "hpq_adjoint_nparams": ([vp, ctypes.POINTER(i32)], i32),
        "hpq_n_cell": ([vp, ctypes.POINTER(i32)], i32),
        "hpq_max_step": ([vp, ctypes.POINTER(i32)], i32),
        "hpq_time": ([vp, dp], i32),
        "hpq_diag_count": ([vp, lp], i32),
        "hpq_beam_name": ([vp, i32], cp),
        "hpq_salame_log": ([vp, dp, lp], i32),
        "hpq_adjoint_grad": ([vp, dp, dp, dp], i32),
        "hpq_synchronize": ([vp], i32),
        "hpq_stream": ([vp], vp),
        "hpq_get_counters": ([vp, lp, lp, lp, lp], i32),
        "hpq_set_profiling": ([vp, i32], i32),
        "hpq_get_profile": ([vp, cp, dp, lp], i32),
        "hpq_poisson_dirichlet_noalloc": ([vp, vp, i32, i32, ctypes.c_double, ctypes.c_double, vp], i32),
        "hpq_beam_slice_count": ([vp, i32, i32, lp], i32),
        "hpq_get_beam_slice": ([vp, i32, i32] + [dp] * 7 + [lp], i32),
        "hpq_put_beam_slice": ([vp, i32, i32] + [dp] * 7 + [lp, i64], i32),
        "hpq_set_time": ([vp, ctypes.c_double], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _lp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


BEAM_ATTRS = ("x", "y", "z", "w", "ux", "uy", "uz")
PLASMA_ATTRS = ("x", "y", "w", "ux", "uy", "psi", "x_prev", "y_prev", "ux_half_step",
                "uy_half_step", "psi_half_step", "valid")


INSITU_BEAM = ("sum(w)", "[x]", "[x^2]", "[y]", "[y^2]", "[z]", "[z^2]", "[ux]", "[ux^2]", "[uy]", "[uy^2]",
               "[uz]", "[uz^2]", "[x*ux]", "[y*uy]", "[z*uz]", "[x*uy]", "[y*ux]", "[ux/uz]", "[uy/uz]", "[ga]",
               "[ga^2]")
INSITU_FIELDS = ("[Ex^2]", "[Ey^2]", "[Ez^2]", "[Bx^2]", "[By^2]", "[Bz^2]", "[ExmBy^2]", "[EypBx^2]",
                 "[jz_beam]", "[Ez*jz_beam]")


def split_insitu(what, flat, nz):
    """Flat in-situ array (hpq_get_insitu layout) -> dict of per-slice arrays and totals."""
    names = INSITU_FIELDS if what == "fields" else INSITU_BEAM
    d = {k: flat[i * nz:(i + 1) * nz] for i, k in enumerate(names)}
    off = len(names) * nz
    if what != "fields":
        d["Np"] = flat[off:off + nz]
        off += nz
    d["sum"] = flat[off:]
    return d


class Hipace:
    """One simulation on one GPU, driven through libhpq."""

    def __init__(self, input_text, precision=PLAIN_FP64, graphs=True, deterministic=False):
        self.L = load_library()
        h = ctypes.c_void_p()
        rc = self.L.hpq_create(input_text.encode(), ctypes.byref(h))
        if rc:
            raise HpqError(rc, self.L.hpq_create_error().decode())
        self.h = h
        self._check(self.L.hpq_set_precision(self.h, precision))
        self._check(self.L.hpq_set_graphs(self.h, int(bool(graphs))))
        self._check(self.L.hpq_set_deterministic(self.h, int(bool(deterministic))))
        nc = (ctypes.c_int * 3)()
        self._check(self.L.hpq_n_cell(self.h, nc))
        self.n_cell = [nc[0], nc[1], nc[2]]
        ms = ctypes.c_int()
        self._check(self.L.hpq_max_step(self.h, ctypes.byref(ms)))
        self.max_step = ms.value
        self.diag_type = _string(input_text, "diagnostic.diag_type", "xyz")
        self._diag = []

    def _check(self, rc):
        if rc:
            raise HpqError(rc, self.L.hpq_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.hpq_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # ---- reference driver surface
    def init_data(self):
        self._check(self.L.hpq_init(self.h))

    def evolve(self, first_step=0, last_step=None):
        """Steps first_step .. last_step (default max_step), leaving the loop after the step
        at hipace.max_time like Hipace::Evolve (Hipace.cpp:401-419)."""
        last = self.max_step if last_step is None else last_step
        for s in range(first_step, last + 1):
            if math.isinf(self.time()):
                break
            self.step(s)

    def salame_log(self):
        """(slice, iteration, W) rows of every SALAME iteration since init_data."""
        n = ctypes.c_int64()
        self._check(self.L.hpq_salame_log(self.h, None, ctypes.byref(n)))
        out = np.zeros(n.value)
        self._check(self.L.hpq_salame_log(self.h, _dp(out), ctypes.byref(n)))
        return out.reshape(-1, 3)

    def time(self):
        """Physical time at which the next step starts (+inf after the step at max_time)."""
        t = ctypes.c_double()
        self._check(self.L.hpq_time(self.h, ctypes.byref(t)))
        return t.value

    def step(self, step):
        self._check(self.L.hpq_step(self.h, step))

    def begin_step(self, step):
        self._check(self.L.hpq_begin_step(self.h, step))

    def solve_one_slice(self, islice):
        self._check(self.L.hpq_solve_slice(self.h, islice))

    def end_step(self):
        self._check(self.L.hpq_end_step(self.h))

    # ---- data access
    def set_beam(self, b, beam):
        arrs = [np.ascontiguousarray(beam[k], dtype=np.float64) for k in BEAM_ATTRS]
        ids = beam.get("id")
        ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int64)
        self._check(self.L.hpq_set_beam(self.h, b, *[_dp(a) for a in arrs],
                                        _lp(ids) if ids is not None else None, len(arrs[0])))

    def get_beam(self, b=0, out=None):
        """Beam particles of species b (hpq_get_beam). `out`, optional, is a dict of contiguous
        arrays (float64, "id" int64) at least as long as the beam, e.g. in pinned memory that is
        reused from step to step; the result is then views of its first entries."""
        n = ctypes.c_int64()
        self._check(self.L.hpq_beam_count(self.h, b, ctypes.byref(n)))
        n = n.value
        if out is not None and all(out[k].size >= n and out[k].flags.c_contiguous for k in BEAM_ATTRS + ("id",)):
            res = {k: out[k][:n] for k in BEAM_ATTRS + ("id",)}
        else:
            res = {k: np.empty(n) for k in BEAM_ATTRS}
            res["id"] = np.empty(n, dtype=np.int64)
        self._check(self.L.hpq_get_beam(self.h, b, *[_dp(res[k]) for k in BEAM_ATTRS], _lp(res["id"])))
        return res

    # ---- time-step pipeline hand-off (hipace2_b200/pipeline.py)
    def get_beam_slice(self, b, islice):
        """Particles that slice `islice` of the current (or last) step hands to the next step."""
        n = ctypes.c_int64()
        self._check(self.L.hpq_beam_slice_count(self.h, b, islice, ctypes.byref(n)))
        res = {k: np.empty(n.value) for k in BEAM_ATTRS}
        res["id"] = np.empty(n.value, dtype=np.int64)
        self._check(self.L.hpq_get_beam_slice(self.h, b, islice, *[_dp(res[k]) for k in BEAM_ATTRS], _lp(res["id"])))
        return res

    def put_beam_slice(self, b, islice, beam):
        """Particles of slice `islice` of the current step, received from the previous step."""
        arrs = [np.ascontiguousarray(beam[k], dtype=np.float64) for k in BEAM_ATTRS]
        ids = np.ascontiguousarray(beam["id"], dtype=np.int64)
        self._check(self.L.hpq_put_beam_slice(self.h, b, islice, *[_dp(a) for a in arrs], _lp(ids), len(ids)))

    def set_time(self, t):
        self._check(self.L.hpq_set_time(self.h, float(t)))

    def get_field(self, comp):
        nx, ny, _ = self.n_cell
        out = np.zeros((ny, nx))
        self._check(self.L.hpq_get_field(self.h, comp.encode(), _dp(out)))
        return out

    def set_diag(self, comps):
        self._diag = list(comps)
        self._check(self.L.hpq_set_diag(self.h, " ".join(comps).encode()))

    def get_diag(self, comp):
        """3-D diagnostic of the last step: (nz, ny, nx), or (nz, nx) / (nz, ny) for
        diagnostic.diag_type = xz / yz."""
        nx, ny, nz = self.n_cell
        out = np.zeros(_diag_shape(self.diag_type, nx, ny, nz))
        n = ctypes.c_int64()
        self._check(self.L.hpq_diag_count(self.h, ctypes.byref(n)))
        assert n.value == out.size, (n.value, out.shape)
        self._check(self.L.hpq_get_diag(self.h, comp.encode(), _dp(out)))
        return out

    def get_insitu(self, what):
        """Reduced in-situ diagnostics of the last diagnostic step of a beam or of "fields" (see
        hpq_get_insitu), split into the reference's named arrays."""
        n = ctypes.c_int64()
        self._check(self.L.hpq_insitu_size(self.h, what.encode(), ctypes.byref(n)))
        out = np.zeros(n.value)
        self._check(self.L.hpq_get_insitu(self.h, what.encode(), _dp(out)))
        return split_insitu(what, out, self.n_cell[2])

    def get_plasma(self, sp=0):
        n = ctypes.c_int64()
        self._check(self.L.hpq_plasma_count(self.h, sp, ctypes.byref(n)))
        n = n.value
        out = np.zeros(12 * n)
        self._check(self.L.hpq_get_plasma(self.h, sp, _dp(out)))
        return {k: out[i * n:(i + 1) * n] for i, k in enumerate(PLASMA_ATTRS)}

    def adjoint_nparams(self):
        n = ctypes.c_int()
        self._check(self.L.hpq_adjoint_nparams(self.h, ctypes.byref(n)))
        return n.value

    def adjoint(self, knots, grad=True):
        """Objective of the adjoint configuration for the given knots and, unless grad is False,
        its gradient (hpq_adjoint_grad): returns J or (J, dJ/dknots)."""
        knots = np.ascontiguousarray(knots, dtype=np.float64)
        n = self.adjoint_nparams()
        if knots.size != n:
            raise ValueError("expected %d knot values, got %d" % (n, knots.size))
        g = np.zeros(n) if grad else None
        J = ctypes.c_double(0)
        self._check(self.L.hpq_adjoint_grad(self.h, _dp(knots), _dp(g) if grad else None, ctypes.byref(J)))
        return (J.value, g) if grad else J.value

    def synchronize(self):
        self._check(self.L.hpq_synchronize(self.h))

    def stream(self):
        return self.L.hpq_stream(self.h)

    def set_deterministic(self, on):
        """Bit-identical results run to run (fixed-point deposition, fixed-order reductions)."""
        self._check(self.L.hpq_set_deterministic(self.h, int(bool(on))))

    def set_profiling(self, on):
        self._check(self.L.hpq_set_profiling(self.h, int(bool(on))))

    def profile(self, kernel_class):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        self._check(self.L.hpq_get_profile(self.h, kernel_class.encode(), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def counters(self):
        a, b, c, d = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.L.hpq_get_counters(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                            ctypes.byref(d)))
        return {"mg_vcycles": a.value, "slices": b.value, "plasma_pushes": c.value, "kernel_launches": d.value}


def _string(text, key, default):
    v = default
    for line in text.splitlines():
        line = line.split("#")[0]
        if "=" in line and line.split("=")[0].strip() == key:
            v = line.split("=", 1)[1].strip().strip('"')
    return v


def _diag_shape(diag_type, nx, ny, nz):
    return {"xyz": (nz, ny, nx), "xz": (nz, nx), "yz": (nz, ny)}[diag_type]
