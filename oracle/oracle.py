"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the FP64 CPU oracle (oracle/ckmpm_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, as the checker.  It is never on the product path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libckmpm_oracle.so"
PIC_LIB = HERE / "_build" / "libpic_baseline.so"

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        d = C.POINTER(C.c_double)
        f = C.POINTER(C.c_float)
        L.oracle_create.argtypes = [C.c_double, C.POINTER(C.c_int32), C.c_double, C.c_double, C.c_int32, C.c_double]
        L.oracle_create.restype = C.c_void_p
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_add_model.argtypes = [C.c_void_p, C.c_int, d, C.c_int, f, f, C.c_int, C.c_double, C.c_double]
        L.oracle_setup.argtypes = [C.c_void_p]
        L.oracle_set_lame.argtypes = [C.c_void_p, C.c_int, d, d]
        L.oracle_set_velocity.argtypes = [C.c_void_p, C.c_int, d, C.c_int]
        L.oracle_set_rigid.argtypes = [C.c_void_p, C.c_int, C.c_int, d]
        L.oracle_set_boundary_field.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), d]
        L.oracle_set_rigid_velocity.argtypes = [C.c_void_p, d]
        L.oracle_step.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.oracle_step_frame.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]
        L.oracle_get_state.argtypes = [C.c_void_p, C.c_int, d, d, d, d, C.POINTER(C.c_uint8)]
        L.oracle_set_state.argtypes = [C.c_void_p, C.c_int, d, d, d]
        L.oracle_counter.argtypes = [C.c_void_p, C.c_int]
        L.oracle_counter.restype = C.c_int64
        L.oracle_current_dt.argtypes = [C.c_void_p]
        L.oracle_current_dt.restype = C.c_double
        L.oracle_get_grid.argtypes = [C.c_void_p, C.POINTER(C.c_int64), d, C.c_int]
        L.oracle_get_blocks.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_uint32),
                                        C.c_int]
        L.oracle_svd3.argtypes = [d, d, d, d]
        L.oracle_ck_w0.argtypes = [C.c_double]
        L.oracle_ck_w0.restype = C.c_double
        L.oracle_constitutive.argtypes = [C.c_int, d, d, C.c_double, d, d, d]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _f(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


class OracleScene:
    """FP64 restatement of the reference substep for one scene (see ckmpm_oracle.cpp)."""

    def __init__(self, config, models=None):
        L = lib()
        dims = (C.c_int32 * 3)(*config.domain_blocks)
        boundary = {"sticky_blocks": 0, "slip_floor": 1, "field": 2}[config.boundary]
        self._h = C.c_void_p(L.oracle_create(config.dx, dims, config.gravity, config.mass_clamp, boundary,
                                             config.floor_cells))
        self.n = []
        if config.boundary == "field" and getattr(config, "boundary_field", None) is not None:
            self.set_boundary_field(*config.boundary_field)
        for m in models or []:
            self.add_model(m)

    def set_boundary_field(self, rule, param=None) -> None:
        """Per-cell boundary rules (x-major over the domain's cells) of a 'field' scene."""
        r = np.ascontiguousarray(rule, np.uint8).ravel()
        p = None if param is None else np.ascontiguousarray(param, np.float64).reshape(-1)
        assert lib().oracle_set_boundary_field(self._h, r.ctypes.data_as(C.POINTER(C.c_uint8)), _d(p)) == 0

    def add_model(self, m) -> int:
        x = np.ascontiguousarray(m.particle_position, np.float32)
        v = np.ascontiguousarray(m.particle_velocity, np.float32)
        p = np.zeros(8, np.float64)
        p[:len(m.material.params())] = m.material.params()
        idx = lib().oracle_add_model(self._h, m.material.kind_code, _d(p), len(x), _f(x), _f(v), len(v),
                                     m.particle_mass, m.particle_volume)
        self.n.append(len(x))
        return idx

    def set_lame(self, model: int, lam, mu) -> None:
        """Per-particle Lame parameters for a fixed-corotated model (None restores the model's own)."""
        if lam is None:
            rc = lib().oracle_set_lame(self._h, model, None, None)
        else:
            lam = np.ascontiguousarray(lam, np.float64)
            mu = np.ascontiguousarray(mu, np.float64)
            rc = lib().oracle_set_lame(self._h, model, _d(lam), _d(mu))
        assert rc == 0

    def set_initial_velocity(self, model: int, v) -> None:
        """Initial velocities in double precision (1 or n rows); call before setup()."""
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
        assert lib().oracle_set_velocity(self._h, model, _d(v), len(v)) == 0

    def set_rigid(self, count: int, velocity) -> None:
        """Rigid particles on: the first `count` particles of every von Mises
        model are rigid and move with `velocity`; call before setup()."""
        v = np.ascontiguousarray(velocity, np.float64).reshape(3)
        assert lib().oracle_set_rigid(self._h, 1, int(count), _d(v)) == 0

    def set_rigid_velocity(self, velocity) -> None:
        v = np.ascontiguousarray(velocity, np.float64).reshape(3)
        assert lib().oracle_set_rigid_velocity(self._h, _d(v)) == 0

    def setup(self):
        lib().oracle_setup(self._h)

    def step(self, nsteps: int, dt: float):
        lib().oracle_step(self._h, nsteps, dt)

    def step_frame(self, dt_max: float, cfl: float, frame_time: float) -> int:
        """One frame with the reference's adaptive dt rule; returns the substeps taken."""
        t = C.c_double(getattr(self, "_time", 0.0))
        k = lib().oracle_step_frame(self._h, dt_max, cfl, frame_time, C.byref(t))
        self._time = t.value
        return k

    def state(self, model: int = 0):
        n = self.n[model]
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        F = np.zeros((n, 3, 3))
        aux = np.zeros(n)
        alive = np.zeros(n, np.uint8)
        lib().oracle_get_state(self._h, model, _d(x), _d(v), _d(F), _d(aux), alive.ctypes.data_as(C.POINTER(C.c_uint8)))
        return dict(x=x, v=v, F=F, aux=aux, alive=alive.astype(bool))

    def set_state(self, model: int, x=None, F=None, aux=None):
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        x, F, aux = conv(x), conv(F), conv(aux)
        lib().oracle_set_state(self._h, model, _d(x), _d(F), _d(aux))

    def counters(self) -> dict:
        L = lib()
        return {"steps": L.oracle_counter(self._h, 0), "lost": L.oracle_counter(self._h, 1),
                "window_skips": L.oracle_counter(self._h, 2), "grid_blocks": L.oracle_counter(self._h, 3)}

    def grid(self):
        L = lib()
        n = L.oracle_get_grid(self._h, None, None, 0)
        keys = np.zeros(n, np.int64)
        data = np.zeros((n, 4, 2, 64))
        L.oracle_get_grid(self._h, keys.ctypes.data_as(C.POINTER(C.c_int64)), _d(data), n)
        return keys, data

    def blocks(self, model: int = -1, which: int = 0):
        L = lib()
        n = L.oracle_get_blocks(self._h, model, which, None, None, 0)
        keys = np.zeros((n, 3), np.int32)
        counts = np.zeros(n, np.uint32)
        L.oracle_get_blocks(self._h, model, which, keys.ctypes.data_as(C.POINTER(C.c_int32)),
                            counts.ctypes.data_as(C.POINTER(C.c_uint32)), n)
        return keys, counts

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def svd3(A):
    A = np.ascontiguousarray(A, np.float64)
    U = np.zeros(9)
    S = np.zeros(3)
    V = np.zeros(9)
    lib().oracle_svd3(_d(A), _d(U), _d(S), _d(V))
    return U.reshape(3, 3), S, V.reshape(3, 3)


def ck_w0(o: float) -> float:
    return lib().oracle_ck_w0(o)


def constitutive(kind: int, params, C_, dt, F, aux):
    p = np.zeros(8, np.float64)
    p[:len(params)] = params
    Cm = np.ascontiguousarray(C_, np.float64).reshape(9)
    Fm = np.ascontiguousarray(F, np.float64).reshape(9).copy()
    a = np.asarray([aux], np.float64)
    tau = np.zeros(9)
    lib().oracle_constitutive(kind, _d(p), _d(Cm), dt, _d(Fm), _d(a), _d(tau))
    return Fm.reshape(3, 3), float(a[0]), tau.reshape(3, 3)
