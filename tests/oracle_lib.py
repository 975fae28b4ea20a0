"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp). Test infrastructure only."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

_lib = None


def build(force=False):
    """Compile the oracle with gcc (recipe in oracle/Makefile)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest_source():
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return LIB


def _newest_source():
    srcs = [os.path.join(ROOT, "oracle", "oracle.cpp"),
            os.path.join(ROOT, "hipace2_b200", "csrc", "config.hpp"),
            os.path.join(ROOT, "hipace2_b200", "csrc", "inputs.hpp"),
            os.path.join(ROOT, "hipace2_b200", "csrc", "rng.hpp")]
    return max(os.path.getmtime(s) for s in srcs)


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, cp, i32, i64 = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int64
        dp = ctypes.POINTER(ctypes.c_double)
        lp = ctypes.POINTER(ctypes.c_int64)
        L.oracle_create.argtypes = [cp, ctypes.POINTER(vp), cp, i32]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_init_beams.argtypes = [vp]
        L.oracle_set_beam.argtypes = [vp, i32] + [dp] * 7 + [lp, i64]
        L.oracle_beam_count.argtypes = [vp, i32]
        L.oracle_beam_count.restype = i64
        L.oracle_get_beam.argtypes = [vp, i32] + [dp] * 7 + [lp]
        L.oracle_set_diag.argtypes = [vp, cp]
        L.oracle_get_diag.argtypes = [vp, cp, dp]
        L.oracle_insitu_size.argtypes = [vp, cp]
        L.oracle_insitu_size.restype = ctypes.c_longlong
        L.oracle_get_insitu.argtypes = [vp, cp, dp]
        L.oracle_step.argtypes = [vp, i32]
        L.oracle_begin_step.argtypes = [vp, i32]
        L.oracle_solve_slice.argtypes = [vp, i32, i32]
        L.oracle_end_step.argtypes = [vp]
        L.oracle_time.argtypes = [vp]
        L.oracle_time.restype = ctypes.c_double
        L.oracle_poisson_dirichlet.argtypes = [dp, dp, i32, i32, ctypes.c_double, ctypes.c_double]
        L.oracle_poisson_dirichlet.restype = i32
        L.oracle_dst1.argtypes = [dp, dp, i32]
        L.oracle_dst1.restype = i32
        L.oracle_salame_log.argtypes = [vp, dp]
        L.oracle_salame_log.restype = ctypes.c_longlong
        L.oracle_get_field.argtypes = [vp, cp, dp]
        L.oracle_plasma_count.argtypes = [vp, i32]
        L.oracle_plasma_count.restype = i64
        L.oracle_get_plasma.argtypes = [vp, i32, dp]
        L.oracle_mg_iterations.argtypes = [vp]
        L.oracle_mg_iterations.restype = ctypes.c_longlong
        L.oracle_threads.restype = i32
        L.oracle_n_cell.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.oracle_adjoint_nparams.argtypes = [vp]
        L.oracle_adjoint_nparams.restype = i32
        L.oracle_adjoint.argtypes = [vp, dp, dp, dp]
        L.oracle_beam_slice_count.argtypes = [vp, i32, i32]
        L.oracle_beam_slice_count.restype = i64
        L.oracle_get_beam_slice.argtypes = [vp, i32, i32] + [dp] * 7 + [lp]
        L.oracle_put_beam_slice.argtypes = [vp, i32, i32] + [dp] * 7 + [lp, i64]
        L.oracle_set_time.argtypes = [vp, ctypes.c_double]
        L.oracle_shape_factor.argtypes = [i32, i32, ctypes.c_double, i32, dp, dp, ctypes.POINTER(ctypes.c_int)]
        L.oracle_shape_factor.restype = i32
        L.oracle_error.argtypes = [vp]
        L.oracle_error.restype = cp
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _lp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


BEAM_ATTRS = ("x", "y", "z", "w", "ux", "uy", "uz")
PLASMA_ATTRS = ("x", "y", "w", "ux", "uy", "psi", "x_prev", "y_prev", "ux_half_step",
                "uy_half_step", "psi_half_step", "valid")


class Oracle:
    def __init__(self, input_text):
        L = lib()
        self.L = L
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        rc = L.oracle_create(input_text.encode(), ctypes.byref(h), err, 1024)
        if rc != 0:
            raise ValueError(err.value.decode())
        self.h = h
        nc = (ctypes.c_int * 3)()
        L.oracle_n_cell(h, nc)
        self.nx, self.ny, self.nz = nc[0], nc[1], nc[2]
        import hipace2_b200 as hp
        self.diag_type = hp._string(input_text, "diagnostic.diag_type", "xyz")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def init_beams(self):
        rc = self.L.oracle_init_beams(self.h)
        if rc:
            raise RuntimeError("fixed_weight_pdf beams must be set with set_beam before init")

    def set_beam(self, b, beam):
        arrs = [np.ascontiguousarray(beam[k], dtype=np.float64) for k in BEAM_ATTRS]
        ids = beam.get("id")
        ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int64)
        n = len(arrs[0])
        self.L.oracle_set_beam(self.h, b, *[_dp(a) for a in arrs],
                               _lp(ids) if ids is not None else None, n)

    def get_beam_slice(self, b, islice):
        n = self.L.oracle_beam_slice_count(self.h, b, islice)
        out = {k: np.zeros(n) for k in BEAM_ATTRS}
        out["id"] = np.zeros(n, dtype=np.int64)
        self.L.oracle_get_beam_slice(self.h, b, islice, *[_dp(out[k]) for k in BEAM_ATTRS], _lp(out["id"]))
        return out

    def put_beam_slice(self, b, islice, beam):
        arrs = [np.ascontiguousarray(beam[k], dtype=np.float64) for k in BEAM_ATTRS]
        ids = np.ascontiguousarray(beam["id"], dtype=np.int64)
        self.L.oracle_put_beam_slice(self.h, b, islice, *[_dp(a) for a in arrs], _lp(ids), len(ids))

    def set_time(self, t):
        self.L.oracle_set_time(self.h, float(t))

    def get_beam(self, b):
        n = self.L.oracle_beam_count(self.h, b)
        out = {k: np.zeros(n) for k in BEAM_ATTRS}
        out["id"] = np.zeros(n, dtype=np.int64)
        self.L.oracle_get_beam(self.h, b, *[_dp(out[k]) for k in BEAM_ATTRS], _lp(out["id"]))
        return out

    def set_diag(self, names):
        if self.L.oracle_set_diag(self.h, " ".join(names).encode()):
            raise KeyError(names)

    def get_diag(self, name):
        import hipace2_b200 as hp
        out = np.zeros(hp._diag_shape(self.diag_type, self.nx, self.ny, self.nz))
        if self.L.oracle_get_diag(self.h, name.encode(), _dp(out)):
            raise KeyError(name)
        return out

    def get_insitu(self, what):
        """Flat in-situ array in the layout of hpq_get_insitu."""
        n = self.L.oracle_insitu_size(self.h, what.encode())
        if n < 0:
            raise KeyError(what)
        out = np.zeros(n)
        if self.L.oracle_get_insitu(self.h, what.encode(), _dp(out)):
            raise KeyError(what)
        return out

    def step(self, s):
        return self.L.oracle_step(self.h, s)

    def begin_step(self, s):
        self.L.oracle_begin_step(self.h, s)

    def solve_slice(self, islice, step):
        return self.L.oracle_solve_slice(self.h, islice, step)

    def end_step(self):
        self.L.oracle_end_step(self.h)

    def time(self):
        return self.L.oracle_time(self.h)

    def salame_log(self):
        """(slice, iteration, W) rows of every SALAME iteration so far."""
        n = self.L.oracle_salame_log(self.h, None)
        out = np.zeros(n)
        self.L.oracle_salame_log(self.h, _dp(out))
        return out.reshape(-1, 3)

    def get_field(self, name):
        out = np.zeros((self.ny, self.nx))
        if self.L.oracle_get_field(self.h, name.encode(), _dp(out)):
            raise KeyError(name)
        return out

    def get_plasma(self, sp=0):
        n = self.L.oracle_plasma_count(self.h, sp)
        out = np.zeros(12 * n)
        self.L.oracle_get_plasma(self.h, sp, _dp(out))
        return {k: out[i * n:(i + 1) * n] for i, k in enumerate(PLASMA_ATTRS)}

    def adjoint(self, theta, grad=True):
        """Objective (and gradient) of the adjoint configuration for parameters theta."""
        n = self.L.oracle_adjoint_nparams(self.h)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        assert theta.size == n, (theta.size, n)
        g = np.zeros(n) if grad else None
        J = ctypes.c_double(0)
        rc = self.L.oracle_adjoint(self.h, _dp(theta), _dp(g) if grad else None, ctypes.byref(J))
        if rc != 0:
            raise RuntimeError("oracle_adjoint failed: %d" % rc)
        return (J.value, g) if grad else J.value

    def mg_iterations(self):
        return self.L.oracle_mg_iterations(self.h)

