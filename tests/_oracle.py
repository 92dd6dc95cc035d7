"""ctypes loader of the CPU oracle (oracle/liboracle.so) -- test infrastructure.

The oracle restates the reference's Fortran routines in C; tests use it only as
the checker of the CUDA library.
"""
from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

from dumses_hybrid_b200 import DgParams, Params

ROOT = pathlib.Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
LIB = ORACLE_DIR / "liboracle.so"

_lib = None


def build_oracle() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "liboracle.so"], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(str(LIB))
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.or_create.restype, L.or_create.argtypes = vp, [ctypes.POINTER(DgParams)]
        L.or_destroy.restype, L.or_destroy.argtypes = None, [vp]
        L.or_uin.restype, L.or_uin.argtypes = dp, [vp]
        L.or_uin_size.restype, L.or_uin_size.argtypes = ctypes.c_longlong, [vp]
        L.or_compute_dt.restype, L.or_compute_dt.argtypes = ctypes.c_double, [vp]
        L.or_godunov.restype, L.or_godunov.argtypes = None, [vp, ctypes.c_double, ctypes.c_double]
        L.or_fargo_update.restype, L.or_fargo_update.argtypes = None, [vp, ctypes.c_double]
        L.or_boundary.restype, L.or_boundary.argtypes = None, [vp, ctypes.c_double, ctypes.c_double]
        L.or_history_mri.restype, L.or_history_mri.argtypes = None, [vp, dp]
        L.or_history_default.restype, L.or_history_default.argtypes = None, [vp, dp]
        L.or_history_1d.restype, L.or_history_1d.argtypes = None, [vp, dp]
        L.or_step.restype, L.or_step.argtypes = ctypes.c_double, [vp, dp]
        L.or_dissipation.restype, L.or_dissipation.argtypes = None, [vp, ctypes.c_double, ctypes.c_double]
        L.or_run_history.restype = ctypes.c_int
        L.or_run_history.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp, ctypes.c_int]
        L.or_array.restype, L.or_array.argtypes = dp, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        L.or_set_threads.restype, L.or_set_threads.argtypes = None, [ctypes.c_int]
        L.or_condinit.restype = ctypes.c_int
        L.or_condinit.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong]
        _lib = L
    return _lib


class _State:
    """Owner of one C oracle state: freed when the last holder (the Oracle, or a view of its
    uin) goes, or by close()."""

    def __init__(self, L, params: Params):
        self.L = L
        self.cp = params.to_c()
        self.h = L.or_create(ctypes.byref(self.cp))

    def close(self):
        if self.h:
            self.L.or_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class _Memory:
    """n doubles of oracle memory at ptr, exposed to numpy with a reference to their owner."""

    def __init__(self, owner: _State, ptr: int, n: int):
        self.owner = owner
        self.__array_interface__ = {"data": (ptr, False), "shape": (n,), "typestr": "<f8", "version": 3}


class Oracle:
    """One oracle state, driven like the reference's module globals.  `uin` is the oracle's
    own memory; views of it keep the state alive until they go (close() frees it at once)."""

    def __init__(self, params: Params):
        self.params = params
        self.L = lib()
        self._state = _State(self.L, params)
        n = self.L.or_uin_size(self.h)
        ptr = ctypes.cast(self.L.or_uin(self.h), ctypes.c_void_p).value
        self.uin = np.asarray(_Memory(self._state, ptr, n)).reshape(params.shape, order="F")

    @property
    def h(self):
        return self._state.h

    def close(self):
        self._state.close()

    def set_state(self, u: np.ndarray) -> None:
        self.uin[...] = u

    def condinit(self, ic: str, beta: float = 1000.0, amp: float = 0.0, seed: int = 0) -> None:
        """Write one of the library's initial conditions into uin (the oracle's own copy of
        the problem set-up, equal bit for bit to dumses_hybrid_b200.condinit)."""
        from dumses_hybrid_b200 import IC
        rc = self.L.or_condinit(self.h, IC[ic], beta, amp, seed)
        if rc != 0:
            raise ValueError(f"or_condinit({ic!r}) returned {rc}")

    def compute_dt(self) -> float:
        return self.L.or_compute_dt(self.h)

    def godunov(self, dt: float, time: float) -> None:
        self.L.or_godunov(self.h, dt, time)

    def fargo_update(self, dt: float) -> None:
        self.L.or_fargo_update(self.h, dt)

    def boundary(self, time: float, dt: float) -> None:
        self.L.or_boundary(self.h, time, dt)

    def dissipation(self, time: float, dt: float) -> None:
        self.L.or_dissipation(self.h, time, dt)

    def step(self, time: float) -> tuple[float, float]:
        t = ctypes.c_double(time)
        dt = self.L.or_step(self.h, ctypes.byref(t))
        return t.value, dt

    def history(self, variant: str = "mri") -> np.ndarray:
        """The 9 history sums: variant "mri" (src/problem/mri/history.f90) or "default"
        (src/subroutines/history.f90); "1d": the one-dimensional line of the default routine
        (rho, rho u_x, E at x = 1/2)."""
        if variant == "1d":
            out = np.zeros(3)
            self.L.or_history_1d(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            return out
        out = np.zeros(9)
        f = self.L.or_history_mri if variant == "mri" else self.L.or_history_default
        f(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def run_history(self, tlim: float, dthist: float, max_rows: int) -> np.ndarray:
        rows = np.zeros((max_rows, 11))
        n = self.L.or_run_history(self.h, tlim, dthist, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), max_rows)
        return rows[:n]

    def array(self, which: int) -> np.ndarray:
        n = ctypes.c_longlong()
        p = self.L.or_array(self.h, which, ctypes.byref(n))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()
