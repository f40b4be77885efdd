"""Host-side mirror of the reference's subroutine interface.

``BGK3D`` exposes the reference's per-rank call sequence
(SRC/bgk3d_HIT.F90:74-146) as methods with the same names:

    input / hencol / alloca  -> BGK3D(...) or BGK3D.from_input("bgk.input")
    init                     -> init()                 (Taylor-Green, SRC/init.F90)
    boundaries(itime)        -> boundaries(itime)      (no-op: wrap in kernel)
    col_MC(itime)            -> col_MC(itime)
    diagnostic(itime, ...)   -> diagnostic(itime)      (gated by icheck)
    diagno(itime)            -> diagno(itime)
    dissipation(itime)       -> dissipation(itime)

``run_loop`` replays the program's time loop and writes ``diagno.dat``
(fort.70, SRC/diagno.F90:137) and ``dissipation.dat`` (fort.71,
SRC/dissipation.F90:261-269) with the reference's columns and formats.

Every call goes through the C-ABI of ``libbgk3d.so``; nothing is computed on
the host.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

from . import _abi
from ._abi import BgkDiag, BgkParams, check

_STORE_DTYPES = {_abi.BGK_FP64: np.float64, _abi.BGK_FP32DEV: np.float32, _abi.BGK_FP16DEV: np.float16}


def read_namelist(path: str) -> dict:
    """Reads the reference's ``&parameters`` namelist (SRC/input.F90:41-47)."""
    text = open(path).read()
    m = re.search(r"&parameters(.*?)/", text, re.S | re.I)
    if not m:
        raise ValueError(f"no &parameters group in {path}")
    out = {}
    for key, val in re.findall(r"(\w+)\s*=\s*([^,\s/]+)", m.group(1)):
        v = val.strip().rstrip(",").replace("d", "e").replace("D", "e")
        try:
            out[key.lower()] = int(v)
        except ValueError:
            out[key.lower()] = float(v)
    return out


class BGK3D:
    """One periodic D3Q19 box on one GPU, driven like the reference program."""

    def __init__(self, lx: int = 64, ly: int | None = None, lz: int | None = None, *, svisc: float = 0.01,
                 u0: float = 0.05, precision: str = "fp64", scheme: str = "two_lattice", icheck: int = 10,
                 mode: str = "corrected", fp16_scale: float = 0.0, device: int = 0, omega: float | None = None,
                 extras: bool = True, kernel: int = 0, les_cs: float = 0.0, proc_z: int = 1, coord_z: int = 0):
        self._lib = _abi.load()
        p = BgkParams()
        check(self._lib.bgk_params_default(C.byref(p)), "bgk_params_default")
        p.lx, p.ly, p.lz = lx, ly or lx, lz or lx
        p.svisc, p.u0 = svisc, u0
        p.precision = _abi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p.scheme = _abi.SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)
        p.mode = _abi.MODES[mode] if isinstance(mode, str) else int(mode)
        p.icheck, p.fp16_scale, p.device, p.extras, p.kernel = icheck, fp16_scale, device, int(extras), kernel
        p.les_cs, p.proc_z, p.coord_z = les_cs, proc_z, coord_z
        if omega is not None:
            p.use_omega, p.omega = 1, omega
        self.params = p
        self._h = C.c_void_p()
        check(self._lib.bgk_create(C.byref(p), C.byref(self._h)), "bgk_create")
        # local shape: a z-slab (proc_z > 1) holds lz/proc_z planes
        self.shape = (p.lx, p.ly, p.lz // max(proc_z, 1))
        self.global_shape = (p.lx, p.ly, p.lz)
        self.dtype = _STORE_DTYPES[p.precision]

    # ----------------------------------------------------------- set-up
    @classmethod
    def from_input(cls, path: str, **kw) -> "BGK3D":
        """input + hencol + alloca from a bgk.input namelist (one rank)."""
        nl = read_namelist(path)
        for ax in ("x", "y"):
            if nl.get("proc_" + ax, 1) != 1:
                raise ValueError("the box is split along z only: proc_x = proc_y = 1")
        kw.setdefault("proc_z", nl.get("proc_z", 1))
        return cls(nl["lx"], nl["ly"], nl["lz"], svisc=nl["svisc"], u0=nl["u0"], icheck=nl.get("icheck", 100), **kw)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bgk_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self) -> int:
        lx, ly, lz = self.shape
        return lx * ly * lz

    def init(self):
        """Taylor-Green vortex (SRC/init.F90:23-163)."""
        check(self._lib.bgk_init_tgv(self._h), "bgk_init_tgv")

    def init_velocity(self, u, v, w, rho: float = 1.0):
        lx, ly, lz = self.shape
        a = [np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(lz, ly, lx)) for x in (u, v, w)]
        dp = C.POINTER(C.c_double)
        check(self._lib.bgk_init_velocity(self._h, a[0].ctypes.data_as(dp), a[1].ctypes.data_as(dp),
                                          a[2].ctypes.data_as(dp), rho), "bgk_init_velocity")

    def init_velocity_device(self, u, v, w, rho: float = 1.0):
        """Equilibrium from a velocity field already on the box's GPU: three
        contiguous float64 torch tensors of shape (lz, ly, lx), read in place
        (bgk_init_velocity_device)."""
        lx, ly, lz = self.shape
        for t in (u, v, w):
            if tuple(t.shape) != (lz, ly, lx) or str(t.dtype) != "torch.float64" or not t.is_contiguous():
                raise ValueError(f"expected contiguous float64 tensors of shape {(lz, ly, lx)}")
        check(self._lib.bgk_init_velocity_device(self._h, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                                 C.c_void_p(w.data_ptr()), rho), "bgk_init_velocity_device")

    # -------------------------------------------------------- time loop
    def boundaries(self, itime: int):
        check(self._lib.bgk_boundaries(self._h, itime), "bgk_boundaries")

    def col_MC(self, itime: int):
        check(self._lib.bgk_col_mc(self._h, itime), "bgk_col_mc")

    def run(self, nsteps: int):
        check(self._lib.bgk_run(self._h, nsteps), "bgk_run")

    def diagnostic(self, itime: int) -> dict | None:
        """Gated like SRC/diagnostic.F90:37: None when mod(itime, icheck) != 0."""
        d = BgkDiag()
        rc = check(self._lib.bgk_diagnostic(self._h, itime, C.byref(d)), "bgk_diagnostic",
                   ok=(_abi.BGK_OK, _abi.BGK_SKIPPED))
        return None if rc == _abi.BGK_SKIPPED else d.as_dict()

    def diagno(self, itime: int) -> np.ndarray:
        out = np.zeros(5)
        check(self._lib.bgk_diagno(self._h, itime, out.ctypes.data_as(C.POINTER(C.c_double))), "bgk_diagno")
        return out

    def dissipation(self, itime: int) -> np.ndarray:
        out = np.zeros(4)
        check(self._lib.bgk_dissipation(self._h, itime, out.ctypes.data_as(C.POINTER(C.c_double))),
              "bgk_dissipation")
        return out

    # ------------------------------------------------------------ data
    def populations(self) -> np.ndarray:
        lx, ly, lz = self.shape
        out = np.empty((19, lz, ly, lx), dtype=self.dtype)
        check(self._lib.bgk_get_populations(self._h, out.ctypes.data), "bgk_get_populations")
        return out

    def set_populations(self, pops: np.ndarray):
        lx, ly, lz = self.shape
        a = np.ascontiguousarray(np.asarray(pops, dtype=self.dtype).reshape(19, lz, ly, lx))
        check(self._lib.bgk_put_populations(self._h, a.ctypes.data), "bgk_put_populations")

    def deviations(self) -> np.ndarray:
        lx, ly, lz = self.shape
        out = np.empty((19, lz, ly, lx), dtype=np.float64)
        check(self._lib.bgk_get_deviations(self._h, out.ctypes.data_as(C.POINTER(C.c_double))),
              "bgk_get_deviations")
        return out

    def velocity(self):
        lx, ly, lz = self.shape
        u, v, w = (np.empty((lz, ly, lx)) for _ in range(3))
        dp = C.POINTER(C.c_double)
        check(self._lib.bgk_get_velocity(self._h, u.ctypes.data_as(dp), v.ctypes.data_as(dp),
                                         w.ctypes.data_as(dp)), "bgk_get_velocity")
        return u, v, w

    def spectrum(self, nbins: int | None = None) -> np.ndarray:
        nb = nbins or (max(self.shape) // 2 + 1)
        out = np.zeros(nb)
        check(self._lib.bgk_spectrum(self._h, nb, out.ctypes.data_as(C.POINTER(C.c_double))), "bgk_spectrum")
        return out

    # ---------------------------------------------------- files (I/O)
    def save(self, path: str):
        """Checkpoint of the populations (restart data)."""
        check(self._lib.bgk_save(self._h, os.fsencode(path)), "bgk_save")

    def load(self, path: str):
        check(self._lib.bgk_load(self._h, os.fsencode(path)), "bgk_load")

    def vtk_xy_bin(self, itime: int, k0: int, out_dir: str = "."):
        """= vtk_xy_bin(itime, k0) (SRC/vtk_xy.binary.F90)."""
        check(self._lib.bgk_vtk(self._h, itime, 1, k0, os.fsencode(out_dir)), "bgk_vtk")

    def vtk_xz_bin(self, itime: int, j0: int, out_dir: str = "."):
        check(self._lib.bgk_vtk(self._h, itime, 2, j0, os.fsencode(out_dir)), "bgk_vtk")

    def vtk_yz_bin(self, itime: int, i0: int, out_dir: str = "."):
        check(self._lib.bgk_vtk(self._h, itime, 3, i0, os.fsencode(out_dir)), "bgk_vtk")

    def vtk_3d_bin(self, itime: int, out_dir: str = "."):
        check(self._lib.bgk_vtk(self._h, itime, 0, 0, os.fsencode(out_dir)), "bgk_vtk")

    # ------------------------------------------------------- properties
    def _getd(self, fn):
        v = C.c_double()
        check(getattr(self._lib, fn)(self._h, C.byref(v)), fn)
        return v.value

    def _getll(self, fn):
        v = C.c_longlong()
        check(getattr(self._lib, fn)(self._h, C.byref(v)), fn)
        return v.value

    @property
    def omega(self) -> float:
        return self._getd("bgk_get_omega")

    @property
    def scale(self) -> float:
        return self._getd("bgk_get_scale")

    @property
    def step(self) -> int:
        return self._getll("bgk_get_step")

    @property
    def device_bytes(self) -> int:
        return self._getll("bgk_get_device_bytes")

    @property
    def launch_count(self) -> int:
        return self._getll("bgk_get_launch_count")

    @property
    def stream(self) -> int:
        return self._lib.bgk_get_stream(self._h) or 0

    def synchronize(self):
        check(self._lib.bgk_synchronize(self._h), "bgk_synchronize")

    def record_event(self):
        """Marks the work queued so far on this context's stream."""
        check(self._lib.bgk_record_event(self._h), "bgk_record_event")

    def wait_event(self, other: "BGK3D"):
        """This context's later work waits for `other`'s last marked work."""
        check(self._lib.bgk_wait_event(self._h, other._h), "bgk_wait_event")

    # ---------------------------------------------------------- z-slabs
    # The halo exchange of SRC/bcond.comm.step3.F90 for a box split along z
    # (proc_z > 1); the orchestration across slabs is in slabs.py.
    def halo_buffer(self) -> tuple[int, int]:
        ptr, n = C.c_void_p(), C.c_size_t()
        check(self._lib.bgk_halo_buffer(self._h, C.byref(ptr), C.byref(n)), "bgk_halo_buffer")
        return ptr.value, n.value

    def halo_ipc_handle(self) -> bytes:
        buf = C.create_string_buffer(64)
        check(self._lib.bgk_halo_ipc_handle(self._h, buf), "bgk_halo_ipc_handle")
        return buf.raw

    def halo_ipc_open(self, handle: bytes) -> int:
        ptr = C.c_void_p()
        check(self._lib.bgk_halo_ipc_open(self._h, C.create_string_buffer(bytes(handle), 64), C.byref(ptr)),
              "bgk_halo_ipc_open")
        return ptr.value

    def halo_connect(self, below: int, above: int):
        check(self._lib.bgk_halo_connect(self._h, C.c_void_p(below), C.c_void_p(above)), "bgk_halo_connect")

    def halo_prime(self):
        check(self._lib.bgk_halo_prime(self._h), "bgk_halo_prime")

    def slab_edge_time_us(self) -> float:
        """Device time of the last step's edge-plane kernel (z-slab)."""
        v = C.c_double()
        check(self._lib.bgk_slab_edge_time(self._h, C.byref(v)), "bgk_slab_edge_time")
        return v.value


def fortran_e(x: float) -> str:
    """Fortran E14.6 edit descriptor (0.ddddddE+ee, right-justified), the
    number format of diagno.dat and dissipation.dat."""
    x = float(x)
    if not np.isfinite(x):
        return "%14s" % ("NaN" if np.isnan(x) else ("Infinity" if x > 0 else "-Infinity"))
    if x == 0.0:
        return "%14s" % "0.000000E+00"
    s = "%.5E" % abs(x)
    e = int(s[8:]) + 1
    body = "%s0.%s%sE%s%02d" % ("-" if x < 0 else "", s[0], s[2:7], "-" if e < 0 else "+", abs(e))
    return "%14s" % body


def run_loop(box: BGK3D, itfin: int, out_dir: str | None = None, itstart: int = 1, ivtim: int | None = None,
             itsave: int | None = None):
    """Replays the time loop of SRC/bgk3d_HIT.F90:127-146 (boundaries, col_MC,
    diagnostic) and returns the diagnostic records; with out_dir, writes
    diagno.dat and dissipation.dat in the reference's formats (i8, e14.6).
    With ivtim, also the three mid-box VTK slices at itime 0 and on every
    diagnostic step that is a multiple of ivtim (SRC/bgk3d_HIT.F90:118-120,
    SRC/diagnostic.F90:52-58); with itsave, a checkpoint every itsave steps."""
    lx, ly, lz = box.shape
    recs = []

    def slices(it):
        box.vtk_xy_bin(it, lz // 2, out_dir)
        box.vtk_xz_bin(it, ly // 2, out_dir)
        box.vtk_yz_bin(it, lx // 2, out_dir)

    if out_dir:
        os.makedirs(out_dir, exist_ok=True)
        if ivtim:
            slices(0)
    for itime in range(itstart, itfin + 1):
        box.boundaries(itime)
        box.col_MC(itime)
        d = box.diagnostic(itime)
        if d is not None:
            recs.append(d)
            if out_dir and ivtim and itime % ivtim == 0:
                slices(itime)
        if out_dir and itsave and itime % itsave == 0:
            box.save(os.path.join(out_dir, "restart.%08d.bin" % itime))
    if out_dir:
        with open(os.path.join(out_dir, "diagno.dat"), "w") as f70, \
                open(os.path.join(out_dir, "dissipation.dat"), "w") as f71:
            for d in recs:
                # format 1004: i8, 5(e14.6,1x) -- itime, xtot, ytot, ztot, rtot, stot
                # (SRC/diagno.F90:137,152); i8, 4(e14.6,1x) (SRC/dissipation.F90:265-278)
                f70.write("%8d" % d["itime"] + "".join(fortran_e(x) + " " for x in (
                    d["ux_mean"], d["uy_mean"], d["uz_mean"], d["rho_mean"], d["ke_mean"])) + "\n")
                f71.write("%8d" % d["itime"] + "".join(fortran_e(x) + " " for x in (
                    d["t"], d["tke_norm"], d["diss"])) + "\n")
    return recs
