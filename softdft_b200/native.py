"""ctypes binding of libsoftdft.so, the device solve behind include/softdft.h.

The library is built in-tree (``__graft_entry__.build()``); importing this
module never falls back to anything else: a missing library or a missing GPU
raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .host.descriptor import Descriptor, Numerics, SolverState

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsoftdft.so")
_LIB = None

SDFT_OK = 0
SDFT_MAX_ITERS = 1
SDFT_ERR_UNSUPPORTED = 3
STATUS_NAMES = {0: "OK", 1: "MAX_ITERS", 2: "ERR_ARG", 3: "ERR_UNSUPPORTED", 4: "ERR_CUDA", 5: "ERR_OOM",
                6: "ERR_NORM", 7: "ERR_NONFINITE", 8: "ERR_TIMEOUT"}
EXPORTS = ["sdft_abi_version", "sdft_last_error", "sdft_device_count", "sdft_numerics_default",
           "sdft_request_create", "sdft_request_destroy", "sdft_request_sizes", "sdft_set_state",
           "sdft_get_state", "sdft_objective", "sdft_solve", "sdft_get_densities", "sdft_grand_potential",
           "sdft_num_species", "sdft_solve_batch", "sdft_last_batch_stats", "sdft_server_create",
           "sdft_server_destroy", "sdft_server_submit", "sdft_server_step", "sdft_server_poll", "sdft_bulk_eval",
           "sdft_grid_supported", "sdft_input_from_yaml", "sdft_input_descriptor", "sdft_input_numerics",
           "sdft_input_bulk_stats", "sdft_input_destroy", "sdft_get_solver_state", "sdft_set_solver_state",
           "sdft_solve_resume", "sdft_anderson_step", "sdft_request_prepare", "sdft_server_set_reserve",
           "sdft_request_resident", "sdft_release_cached_memory", "sdft_server_set_pipeline"]


class SdftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def release_cached_memory() -> int:
    """Return the device blocks that the library caches from destroyed requests
    to the driver (sdft_release_cached_memory); the number of bytes released."""
    b = C.c_int64()
    _check(lib().sdft_release_cached_memory(C.byref(b)))
    return int(b.value)


def grid_supported(np_: int) -> bool:
    """True when the device solve runs a grid of np_ points (sdft_grid_supported)."""
    f = lib().sdft_grid_supported
    f.argtypes = [C.c_int32]
    f.restype = C.c_int
    return f(int(np_)) == SDFT_OK


def library_present() -> bool:
    """True when the shared library has been built next to this module."""
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build the CUDA extension first (__graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.sdft_abi_version.restype = C.c_int32
        L.sdft_last_error.restype = C.c_char_p
        L.sdft_device_count.argtypes = [C.POINTER(C.c_int32)]
        L.sdft_numerics_default.argtypes = [vp]
        L.sdft_numerics_default.restype = None
        L.sdft_request_create.argtypes = [vp, C.c_int32, C.POINTER(vp)]
        L.sdft_request_prepare.argtypes = [vp, C.c_int32, C.POINTER(vp)]
        L.sdft_server_set_reserve.argtypes = [vp, C.c_int64]
        L.sdft_server_set_pipeline.argtypes = [vp, C.c_int32]
        L.sdft_release_cached_memory.argtypes = [C.POINTER(C.c_int64)]
        L.sdft_request_destroy.argtypes = [vp]
        L.sdft_request_sizes.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.sdft_set_state.argtypes = [vp, vp, vp, vp, vp]
        L.sdft_get_state.argtypes = [vp, vp, vp, vp, vp]
        L.sdft_objective.argtypes = [vp, vp, vp, vp, vp]
        L.sdft_solve.argtypes = [vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.sdft_get_densities.argtypes = [vp, vp, vp, vp]
        L.sdft_grand_potential.argtypes = [vp, C.POINTER(C.c_double)]
        L.sdft_num_species.argtypes = [vp, vp]
        L.sdft_solve_batch.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
        L.sdft_last_batch_stats.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int32), vp, C.c_int32]
        L.sdft_server_create.argtypes = [vp, C.c_int32, C.c_int64, C.POINTER(vp)]
        L.sdft_server_destroy.argtypes = [vp]
        L.sdft_server_submit.argtypes = [vp, vp, C.c_int64]
        L.sdft_server_step.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.sdft_server_poll.argtypes = [vp, vp, vp, vp, vp, vp, C.c_int32, C.POINTER(C.c_int32)]
        L.sdft_get_solver_state.argtypes = [vp, vp, vp, vp]
        L.sdft_set_solver_state.argtypes = [vp, vp, vp, vp]
        L.sdft_solve_resume.argtypes = [vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.sdft_anderson_step.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(C.c_double)]
        _LIB = L
    return _LIB


def _check(rc: int) -> int:
    if rc not in (SDFT_OK, SDFT_MAX_ITERS):
        raise SdftError(rc, lib().sdft_last_error().decode())
    return rc


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def device_count() -> int:
    c = C.c_int32()
    lib().sdft_device_count(C.byref(c))
    return int(c.value)


class DeviceSystem:
    """One request on the GPU (the C-ABI handle).  With prepare=True the
    request takes no device memory until it is first used or a server admits
    it (sdft_request_prepare)."""

    def __init__(self, d: Descriptor, precision: int = 0, prepare: bool = False):
        self.d = d
        self.h = C.c_void_p()
        make = lib().sdft_request_prepare if prepare else lib().sdft_request_create
        _check(make(C.byref(d.desc), precision, C.byref(self.h)))
        n = C.c_int64()
        b = C.c_int64()
        lib().sdft_request_sizes(self.h, C.byref(n), C.byref(b))
        self.n = int(n.value)
        self.device_bytes = int(b.value)

    def close(self):
        if self.h:
            lib().sdft_request_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _split(self, x):
        d = self.d
        P, NB, MB = d.np_, d.nb, d.mb
        return (x[: P * NB], x[P * NB: P * (NB + 2 * MB)], x[P * (NB + 2 * MB): P * (NB + 2 * MB + 1)], x[-1:])

    def get_x(self) -> np.ndarray:
        x = np.zeros(self.n)
        mu, lng, psi, psic = self._split(x)
        _check(lib().sdft_get_state(self.h, _p(mu), _p(lng) if lng.size else None, _p(psi), _p(psic)))
        return x

    def set_x(self, x: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        mu, lng, psi, psic = (np.ascontiguousarray(a) for a in self._split(x))
        _check(lib().sdft_set_state(self.h, _p(mu), _p(lng) if lng.size else None, _p(psi), _p(psic)))

    def objective(self) -> np.ndarray:
        g = np.zeros(self.n)
        mu, lng, psi, psic = self._split(g)
        _check(lib().sdft_objective(self.h, _p(mu), _p(lng) if lng.size else None, _p(psi), _p(psic)))
        return g

    def solve(self, num: Numerics):
        it = C.c_int32()
        err = C.c_double()
        rc = _check(lib().sdft_solve(self.h, C.byref(num), C.byref(it), C.byref(err)))
        return int(it.value), float(err.value), rc

    def resident(self) -> int:
        """Requests of this shape the device runs at once (sdft_request_resident)."""
        n = C.c_int32()
        f = lib().sdft_request_resident
        f.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        _check(f(self.h, C.byref(n)))
        return int(n.value)

    def solve_resume(self, num: Numerics):
        """Continue the solve from the stored solver state (sdft_solve_resume)."""
        it = C.c_int32()
        err = C.c_double()
        rc = _check(lib().sdft_solve_resume(self.h, C.byref(num), C.byref(it), C.byref(err)))
        return int(it.value), float(err.value), rc

    def solver_state(self):
        """(SolverState, hist_x, hist_g): the driver's scalars and ring buffers
        (anderm columns of n unknowns each)."""
        st = SolverState()
        _check(lib().sdft_get_solver_state(self.h, C.byref(st), None, None))
        m = st.anderm
        hx = np.zeros(max(m, 1) * self.n)
        hg = np.zeros(max(m, 1) * self.n)
        _check(lib().sdft_get_solver_state(self.h, C.byref(st), _p(hx), _p(hg)))
        return st, hx[: m * self.n].reshape(m, self.n), hg[: m * self.n].reshape(m, self.n)

    def set_solver_state(self, st: SolverState, hist_x=None, hist_g=None) -> None:
        hx = None if hist_x is None else np.ascontiguousarray(hist_x, dtype=np.float64).ravel()
        hg = None if hist_g is None else np.ascontiguousarray(hist_g, dtype=np.float64).ravel()
        for a in (hx, hg):
            if a is not None and a.size != st.anderm * self.n:
                raise ValueError("history must hold anderm columns of n unknowns")
        _check(lib().sdft_set_solver_state(self.h, C.byref(st), _p(hx), _p(hg)))

    def anderson_step(self, num: Numerics, g: np.ndarray) -> float:
        """One driver iteration with the caller's G(x) (sdft_anderson_step);
        returns the max-norm residual of the iteration."""
        g = np.ascontiguousarray(g, dtype=np.float64)
        mu, lng, psi, psic = (np.ascontiguousarray(a) for a in self._split(g))
        err = C.c_double()
        _check(lib().sdft_anderson_step(self.h, C.byref(num), _p(mu), _p(lng) if lng.size else None, _p(psi),
                                        _p(psic), C.byref(err)))
        return float(err.value)

    def densities(self):
        d = self.d
        segs = [np.zeros(d.np_ * d.max_states[u] * d.n_seg[u]) for u in range(d.n_species)]
        arr = (C.c_void_p * d.n_species)(*[s.ctypes.data for s in segs])
        beads = np.zeros(d.np_ * d.nb)
        bonds = np.zeros(max(d.np_ * 2 * d.mb, 1))
        _check(lib().sdft_get_densities(self.h, arr, _p(beads), _p(bonds)))
        return segs, beads, bonds[: d.np_ * 2 * d.mb]

    def grand_potential(self) -> float:
        om = C.c_double()
        _check(lib().sdft_grand_potential(self.h, C.byref(om)))
        return float(om.value)

    def num_species(self) -> np.ndarray:
        out = np.zeros(self.d.n_species)
        _check(lib().sdft_num_species(self.h, _p(out)))
        return out


def solve_batch(systems, num: Numerics):
    n = len(systems)
    hs = (C.c_void_p * n)(*[s.h.value for s in systems])
    iters = np.zeros(n, dtype=np.int32)
    errs = np.zeros(n)
    status = np.zeros(n, dtype=np.int32)
    rc = lib().sdft_solve_batch(hs, n, C.byref(num), _p(iters), _p(errs), _p(status))
    if rc not in (0, 1, 6, 7):
        raise SdftError(rc, lib().sdft_last_error().decode())
    return iters, errs, status


def last_batch_stats(n: int = 0):
    """(device_ms, launches, per-request latency ms) of the last solve on this thread."""
    ms = C.c_double()
    launches = C.c_int32()
    lat = np.zeros(max(n, 1))
    lib().sdft_last_batch_stats(C.byref(ms), C.byref(launches), _p(lat), n)
    return float(ms.value), int(launches.value), lat[:n]


def objective_noalloc(d: Descriptor, x_dev_ptr: int, g_dev_ptr: int, stream_ptr: int = 0) -> None:
    """G(x) through sdft_objective_noalloc: no device allocation by the library;
    x and G(x) are the caller's device arrays (n doubles each, raw pointers)."""
    L = lib()
    f = L.sdft_objective_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    _check(f(C.byref(d.desc), C.c_void_p(x_dev_ptr), C.c_void_p(g_dev_ptr), C.c_void_p(stream_ptr or None)))


class Server:
    """Continuous-batching solve server (sdft_server_*): requests are admitted
    into free slots as earlier ones finish; each step is one launch."""

    def __init__(self, num: Numerics, max_slots: int, max_bytes: int = 0):
        self.h = C.c_void_p()
        _check(lib().sdft_server_create(C.byref(num), int(max_slots), int(max_bytes), C.byref(self.h)))
        self._held = {}

    def close(self):
        if self.h:
            lib().sdft_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_reserve(self, reserve_bytes: int) -> None:
        """Device bytes that admission leaves free (sdft_server_set_reserve)."""
        _check(lib().sdft_server_set_reserve(self.h, int(reserve_bytes)))

    def set_pipeline(self, on: bool) -> None:
        """Pipelined stepping (sdft_server_set_pipeline): a step returns once its
        launch is queued, and that launch's finished requests are reported after
        the next step."""
        _check(lib().sdft_server_set_pipeline(self.h, 1 if on else 0))

    def submit(self, system: "DeviceSystem", tag: int) -> None:
        _check(lib().sdft_server_submit(self.h, system.h, int(tag)))
        self._held[int(tag)] = system

    def step(self, iters: int):
        a, q = C.c_int32(), C.c_int32()
        _check(lib().sdft_server_step(self.h, int(iters), C.byref(a), C.byref(q)))
        return int(a.value), int(q.value)

    def poll(self, max_n: int = 4096):
        tags = np.zeros(max_n, dtype=np.int64)
        st = np.zeros(max_n, dtype=np.int32)
        it = np.zeros(max_n, dtype=np.int32)
        err = np.zeros(max_n)
        dms = np.zeros(max_n)
        n = C.c_int32()
        _check(lib().sdft_server_poll(self.h, _p(tags), _p(st), _p(it), _p(err), _p(dms), max_n, C.byref(n)))
        out = []
        for i in range(n.value):
            self._held.pop(int(tags[i]), None)
            out.append((int(tags[i]), int(st[i]), int(it[i]), float(err[i]), float(dms[i])))
        return out


class Input:
    """A request parsed from input.yaml text by the library's host pipeline
    (sdft_input_from_yaml); ``descriptor()`` feeds DeviceSystem."""

    def __init__(self, yaml_text: str):
        L = lib()
        L.sdft_input_from_yaml.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        L.sdft_input_descriptor.restype = C.c_void_p
        L.sdft_input_descriptor.argtypes = [C.c_void_p]
        L.sdft_input_destroy.argtypes = [C.c_void_p]
        self.h = C.c_void_p()
        _check(L.sdft_input_from_yaml(yaml_text.encode(), C.byref(self.h)))

    def descriptor(self):
        from .host.descriptor import Descriptor, SystemDesc
        d = SystemDesc.from_address(lib().sdft_input_descriptor(self.h))
        out = Descriptor(desc=d, keep=[self], np_=d.np, nb=d.nb, mb=d.mb, n_species=d.n_species)
        for u in range(d.n_species):
            sp = d.species[u]
            out.n_seg.append(sp.n_seg)
            out.max_states.append(sp.max_states)
            out.fixed_coord.append(np.ctypeslib.as_array(sp.fixed_coord, (sp.n_seg,)).copy())
            out.mu_species.append(sp.mu_species)
        return out

    def numerics(self):
        from .host.descriptor import Numerics
        n = Numerics()
        _check(lib().sdft_input_numerics(self.h, C.byref(n)))
        return n

    def bulk_stats(self):
        it, res = C.c_int32(), C.c_double()
        _check(lib().sdft_input_bulk_stats(self.h, C.byref(it), C.byref(res)))
        return int(it.value), float(res.value)

    def close(self):
        if self.h:
            lib().sdft_input_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
