"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's Fortran hot path in C (``bgk_oracle.c``).
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only to check results or as the timed CPU baseline.
The product library never loads it.

Parity unpinned: the reference ships no golden vectors and cannot be compiled
in this environment (Fortran + MPI), so the restatement is checked against
itself (ghost-fill vs modulo indexing, conservation, exact rational
arithmetic of a single cell) and against physics known answers.

Array convention (same as the product C-ABI): populations are q-major,
Fortran order within a population (i fastest), i.e. a numpy array of shape
(19, nz, ny, nx) in C order. Values are deviations f - w (times the scale for
the f16 form).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbgk_oracle.so")

_lib = None

_FORMS = {"f64": np.float64, "f32": np.float32, "f16": np.float16}


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(os.path.join(HERE, f)) for f in ("bgk_oracle.c", "bgk_oracle_impl.h")
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        dp = C.POINTER(C.c_double)
        for suf in ("_f64", "_f32", "_f16"):
            f = lambda n: getattr(L, n + suf)  # noqa: E731
            f("orc_create").restype = vp
            f("orc_create").argtypes = [i, i, i]
            f("orc_destroy").argtypes = [vp]
            f("orc_set_scale").argtypes = [vp, d]
            f("orc_set_les").argtypes = [vp, d]
            f("orc_init_tgv").argtypes = [vp, d, i]
            f("orc_init_velocity").argtypes = [vp, dp, dp, dp, d]
            f("orc_boundaries").argtypes = [vp]
            f("orc_omega").restype = d
            f("orc_omega").argtypes = [d]
            f("orc_col_mc_omega").argtypes = [vp, d, i]
            f("orc_col_mc").argtypes = [vp, d, i]
            f("orc_step").argtypes = [vp, d]
            if suf != "_f16":
                f("orc_step_rows").argtypes = [vp, d]
            f("orc_diagno").argtypes = [vp, i, dp]
            f("orc_dissipation").argtypes = [vp, d, d, i, i, dp]
            f("orc_extras").argtypes = [vp, d, dp]
            f("orc_get_pops").argtypes = [vp, vp]
            f("orc_get_dev").argtypes = [vp, dp]
            f("orc_put_pops").argtypes = [vp, vp]
            f("orc_ghost_value").restype = d
            f("orc_ghost_value").argtypes = [vp, i, C.c_long, C.c_long, C.c_long]
        L.orc_num_threads.restype = i
        L.orc_set_num_threads.argtypes = [i]
        L.orc_time_steps_f64.restype = d
        L.orc_time_steps_f64.argtypes = [vp, d, i]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def omega(svisc: float, form: str = "f64") -> float:
    """Collision frequency of SRC/hencol.F90:31 in the form's arithmetic."""
    return getattr(lib(), "orc_omega_" + form)(svisc)


class OracleLattice:
    """Two ghosted D3Q19 lattices, restating the reference's module storage."""

    def __init__(self, nx: int, ny: int, nz: int, form: str = "f64", scale: float = 1.0):
        if form not in _FORMS:
            raise ValueError(form)
        self.form, self.shape = form, (nx, ny, nz)
        self.dtype = _FORMS[form]
        self._L = lib()
        self._s = "_" + form
        self.h = self._f("orc_create")(nx, ny, nz)
        if not self.h:
            raise MemoryError("oracle allocation failed")
        if form == "f16":
            self._f("orc_set_scale")(self.h, scale)
        self.scale = scale

    def _f(self, name):
        return getattr(self._L, name + self._s)

    def close(self):
        if self.h:
            self._f("orc_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    def set_les(self, cs: float):
        """LES collision of SRC/col_MC.F90:221-309 with cteS = cs (0: BGK)."""
        self._f("orc_set_les")(self.h, cs)

    def init_tgv(self, u0: float, faithful: bool = True):
        self._f("orc_init_tgv")(self.h, u0, int(faithful))

    def init_velocity(self, u, v, w, rho: float = 1.0):
        nx, ny, nz = self.shape
        arrs = [np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(nz, ny, nx)) for x in (u, v, w)]
        self._f("orc_init_velocity")(self.h, _dptr(arrs[0]), _dptr(arrs[1]), _dptr(arrs[2]), rho)

    def boundaries(self):
        self._f("orc_boundaries")(self.h)

    def col_mc(self, svisc: float, periodic: bool = False):
        self._f("orc_col_mc")(self.h, svisc, int(periodic))

    def col_mc_omega(self, om: float, periodic: bool = False):
        self._f("orc_col_mc_omega")(self.h, om, int(periodic))

    def step(self, svisc: float, periodic: bool = False):
        """One loop body: boundaries + col_MC (ghost mode) or the modulo form."""
        if periodic:
            self.col_mc(svisc, True)
        else:
            self._f("orc_step")(self.h, svisc)

    def step_rows(self, svisc: float):
        """boundaries + col_MC in the row-vectorised CPU form (bit-identical)."""
        self._f("orc_step_rows")(self.h, svisc)

    def diagno(self, faithful: bool = False) -> np.ndarray:
        out = np.zeros(5)
        self._f("orc_diagno")(self.h, int(faithful), _dptr(out))
        return out

    def dissipation(self, svisc: float, u0: float, itime: int, faithful: bool | int = False) -> np.ndarray:
        """faithful: False/0 periodic pulls, compensated sums; True/1 stale
        ghosts (the reference's), sequential sums; 2 stale ghosts, compensated
        sums."""
        out = np.zeros(4)
        self._f("orc_dissipation")(self.h, svisc, u0, itime, int(faithful), _dptr(out))
        return out

    def extras(self, svisc: float) -> np.ndarray:
        out = np.zeros(3)
        self._f("orc_extras")(self.h, svisc, _dptr(out))
        return out

    def get_pops(self) -> np.ndarray:
        nx, ny, nz = self.shape
        out = np.empty((19, nz, ny, nx), dtype=self.dtype)
        self._f("orc_get_pops")(self.h, out.ctypes.data)
        return out

    def get_dev(self) -> np.ndarray:
        nx, ny, nz = self.shape
        out = np.empty((19, nz, ny, nx), dtype=np.float64)
        self._f("orc_get_dev")(self.h, _dptr(out))
        return out

    def put_pops(self, pops: np.ndarray):
        nx, ny, nz = self.shape
        a = np.ascontiguousarray(np.asarray(pops, dtype=self.dtype).reshape(19, nz, ny, nx))
        self._f("orc_put_pops")(self.h, a.ctypes.data)

    def ghost_value(self, q: int, i: int, j: int, k: int) -> float:
        return self._f("orc_ghost_value")(self.h, q, i, j, k)

    def time_steps(self, svisc: float, steps: int) -> float:
        if self.form != "f64":
            raise ValueError("timed baseline is the f64 form")
        return self._L.orc_time_steps_f64(self.h, svisc, steps)


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int):
    lib().orc_set_num_threads(n)
