"""ctypes binding of liboracle.so -- TEST INFRASTRUCTURE ONLY.

The oracle is the checker of the device solve: tests/, the smoke check and
the CPU-baseline leg of bench.py load it; the product path never does.
Parity status: unpinned (no runnable reference, no reference golden vectors).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from softdft_b200.host.descriptor import Descriptor, Numerics, SolverState

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        L.oracle_create.argtypes = [vp, C.POINTER(vp)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_destroy.restype = None
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_n_unknowns.argtypes = [vp]
        L.oracle_n_unknowns.restype = C.c_int64
        L.oracle_set_x.argtypes = [vp, vp]
        L.oracle_get_x.argtypes = [vp, vp]
        L.oracle_objective.argtypes = [vp, vp]
        L.oracle_solve.argtypes = [vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.oracle_solve_trace.argtypes = [vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_double), vp, C.c_int32]
        L.oracle_get_densities.argtypes = [vp, vp, vp, vp]
        L.oracle_grand_potential.argtypes = [vp, C.POINTER(C.c_double)]
        L.oracle_num_species.argtypes = [vp, vp]
        L.oracle_get_fields.argtypes = [vp, vp, vp]
        L.oracle_solve_many.argtypes = [vp, C.c_int32, vp, vp, vp, vp, C.c_int32]
        L.oracle_max_threads.restype = C.c_int
        L.oracle_get_solver_state.argtypes = [vp, vp, vp, vp]
        L.oracle_set_solver_state.argtypes = [vp, vp, vp, vp]
        L.oracle_solve_resume.argtypes = [vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.oracle_anderson_step.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
        _LIB = L
    return _LIB


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc not in (0, 1):
        raise OracleError(f"oracle status {rc}: {lib().oracle_last_error().decode()}")
    return rc


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleSystem:
    """One system on the CPU oracle; mirrors the device handle's calls."""

    def __init__(self, d: Descriptor):
        self.d = d
        self.h = C.c_void_p()
        _check(lib().oracle_create(C.byref(d.desc), C.byref(self.h)))
        self.n = int(lib().oracle_n_unknowns(self.h))

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_x(self) -> np.ndarray:
        x = np.empty(self.n)
        lib().oracle_get_x(self.h, _p(x))
        return x

    def set_x(self, x: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.size == self.n
        lib().oracle_set_x(self.h, _p(x))

    def objective(self) -> np.ndarray:
        g = np.empty(self.n)
        _check(lib().oracle_objective(self.h, _p(g)))
        return g

    def solve(self, num: Numerics, trace_len: int = 0):
        it = C.c_int32()
        err = C.c_double()
        tr = np.zeros(max(trace_len, 1))
        rc = _check(lib().oracle_solve_trace(self.h, C.byref(num), C.byref(it), C.byref(err), _p(tr), trace_len))
        return int(it.value), float(err.value), rc, tr[: min(trace_len, it.value)]

    def solve_resume(self, num: Numerics):
        it = C.c_int32()
        err = C.c_double()
        rc = _check(lib().oracle_solve_resume(self.h, C.byref(num), C.byref(it), C.byref(err)))
        return int(it.value), float(err.value), rc

    def solver_state(self):
        st = SolverState()
        _check(lib().oracle_get_solver_state(self.h, C.byref(st), None, None))
        hx = np.zeros(st.anderm * self.n)
        hg = np.zeros(st.anderm * self.n)
        _check(lib().oracle_get_solver_state(self.h, C.byref(st), _p(hx), _p(hg)))
        return st, hx.reshape(st.anderm, self.n), hg.reshape(st.anderm, self.n)

    def set_solver_state(self, st: SolverState, hist_x=None, hist_g=None) -> None:
        hx = None if hist_x is None else np.ascontiguousarray(hist_x, dtype=np.float64).ravel()
        hg = None if hist_g is None else np.ascontiguousarray(hist_g, dtype=np.float64).ravel()
        _check(lib().oracle_set_solver_state(self.h, C.byref(st), _p(hx) if hx is not None else None,
                                             _p(hg) if hg is not None else None))

    def anderson_step(self, num: Numerics, g: np.ndarray) -> float:
        g = np.ascontiguousarray(g, dtype=np.float64)
        err = C.c_double()
        _check(lib().oracle_anderson_step(self.h, C.byref(num), _p(g), C.byref(err)))
        return float(err.value)

    def densities(self):
        d = self.d
        segs = [np.zeros(d.np_ * d.max_states[u] * d.n_seg[u]) for u in range(d.n_species)]
        arr = (C.c_void_p * d.n_species)(*[s.ctypes.data for s in segs])
        beads = np.zeros(d.np_ * d.nb)
        bonds = np.zeros(max(d.np_ * 2 * d.mb, 1))
        lib().oracle_get_densities(self.h, arr, _p(beads), _p(bonds))
        return segs, beads, bonds[: d.np_ * 2 * d.mb]

    def grand_potential(self) -> float:
        om = C.c_double()
        _check(lib().oracle_grand_potential(self.h, C.byref(om)))
        return float(om.value)

    def num_species(self) -> np.ndarray:
        out = np.zeros(self.d.n_species)
        lib().oracle_num_species(self.h, _p(out))
        return out

    def fields(self):
        ext = np.zeros(self.d.np_ * self.d.nb)
        tr = np.zeros(self.d.np_ * self.d.nb)
        lib().oracle_get_fields(self.h, _p(ext), _p(tr))
        return ext, tr


def solve_many(systems, num: Numerics, threads: int = 0):
    n = len(systems)
    hs = (C.c_void_p * n)(*[s.h.value for s in systems])
    iters = np.zeros(n, dtype=np.int32)
    errs = np.zeros(n)
    status = np.zeros(n, dtype=np.int32)
    lib().oracle_solve_many(hs, n, C.byref(num), _p(iters), _p(errs), _p(status), threads)
    return iters, errs, status


def max_threads() -> int:
    return int(lib().oracle_max_threads())
