"""ctypes bindings of the C-ABI declared in ``include/bgk3d.h``.

The shared library ``libbgk3d.so`` is built in-tree by ``bgk3d_hit_b200.build``
(nvcc, sm_100a). Loading fails loudly when it is missing: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbgk3d.so")

BGK_OK = 0
BGK_SKIPPED = 1
BGK_ERR_INVALID = -1
BGK_ERR_CUDA = -2
BGK_ERR_NOMEM = -3
BGK_ERR_STATE = -4
BGK_ERR_NONFINITE = -5

BGK_FP64, BGK_FP32DEV, BGK_FP16DEV = 0, 1, 2
BGK_TWO_LATTICE, BGK_AA = 0, 1
BGK_CORRECTED, BGK_FAITHFUL = 0, 1
BGK_ADJ_RECOMPUTE, BGK_ADJ_REBUILD = 0, 1

PRECISIONS = {"fp64": BGK_FP64, "fp32": BGK_FP32DEV, "fp16": BGK_FP16DEV}
SCHEMES = {"two_lattice": BGK_TWO_LATTICE, "aa": BGK_AA}
MODES = {"corrected": BGK_CORRECTED, "faithful": BGK_FAITHFUL}


class BgkParams(C.Structure):
    _fields_ = [
        ("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int),
        ("svisc", C.c_double), ("u0", C.c_double),
        ("precision", C.c_int), ("scheme", C.c_int), ("icheck", C.c_int), ("mode", C.c_int),
        ("fp16_scale", C.c_double), ("device", C.c_int),
        ("use_omega", C.c_int), ("omega", C.c_double), ("extras", C.c_int), ("kernel", C.c_int),
        ("les_cs", C.c_double), ("proc_z", C.c_int), ("coord_z", C.c_int),
    ]


class BgkDiag(C.Structure):
    _fields_ = [
        ("itime", C.c_int),
        ("rho_mean", C.c_double), ("ux_mean", C.c_double), ("uy_mean", C.c_double),
        ("uz_mean", C.c_double), ("ke_mean", C.c_double),
        ("t", C.c_double), ("tke_norm", C.c_double), ("diss", C.c_double), ("tke", C.c_double),
        ("enstrophy", C.c_double), ("eps_strain", C.c_double), ("nonfinite", C.c_longlong),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


# (name, restype, argtypes) for every entry point of include/bgk3d.h
_vp, _i, _d, _ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
_dp = C.POINTER(C.c_double)
PROTOTYPES = [
    ("bgk_params_default", _i, [C.POINTER(BgkParams)]),
    ("bgk_create", _i, [C.POINTER(BgkParams), C.POINTER(_vp)]),
    ("bgk_destroy", _i, [_vp]),
    ("bgk_init_tgv", _i, [_vp]),
    ("bgk_init_velocity", _i, [_vp, _dp, _dp, _dp, _d]),
    ("bgk_init_velocity_device", _i, [_vp, _vp, _vp, _vp, _d]),
    ("bgk_slab_edge_time", _i, [_vp, _dp]),
    ("bgk_boundaries", _i, [_vp, _i]),
    ("bgk_col_mc", _i, [_vp, _i]),
    ("bgk_run", _i, [_vp, _i]),
    ("bgk_diagnostic", _i, [_vp, _i, C.POINTER(BgkDiag)]),
    ("bgk_diagno", _i, [_vp, _i, _dp]),
    ("bgk_dissipation", _i, [_vp, _i, _dp]),
    ("bgk_get_populations", _i, [_vp, _vp]),
    ("bgk_put_populations", _i, [_vp, _vp]),
    ("bgk_get_deviations", _i, [_vp, _dp]),
    ("bgk_get_velocity", _i, [_vp, _dp, _dp, _dp]),
    ("bgk_spectrum", _i, [_vp, _i, _dp]),
    ("bgk_save", _i, [_vp, C.c_char_p]),
    ("bgk_load", _i, [_vp, C.c_char_p]),
    ("bgk_vtk", _i, [_vp, _i, _i, _i, C.c_char_p]),
    ("bgk_adjoint", _i, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _i, _i, _dp, _dp, _dp]),
    ("bgk_adjoint_cache", _i, [_vp, C.c_size_t]),
    ("bgk_adjoint_mode", _i, [_vp, _i]),
    ("bgk_adjoint_rebuilds", _i, [_i, _d, _i]),
    ("bgk_tangent", _i, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _d, _dp, _dp, _dp, _i, _dp, _dp]),
    ("bgk_get_scale", _i, [_vp, _dp]),
    ("bgk_get_omega", _i, [_vp, _dp]),
    ("bgk_get_step", _i, [_vp, C.POINTER(_ll)]),
    ("bgk_get_device_bytes", _i, [_vp, C.POINTER(_ll)]),
    ("bgk_get_launch_count", _i, [_vp, C.POINTER(_ll)]),
    ("bgk_get_stream", _vp, [_vp]),
    ("bgk_synchronize", _i, [_vp]),
    ("bgk_record_event", _i, [_vp]),
    ("bgk_wait_event", _i, [_vp, _vp]),
    ("bgk_halo_buffer", _i, [_vp, C.POINTER(_vp), C.POINTER(C.c_size_t)]),
    ("bgk_halo_ipc_handle", _i, [_vp, _vp]),
    ("bgk_halo_ipc_open", _i, [_vp, _vp, C.POINTER(_vp)]),
    ("bgk_halo_connect", _i, [_vp, _vp, _vp]),
    ("bgk_halo_prime", _i, [_vp]),
    ("bgk_shift3", _i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp]),
    ("bgk_diagnostics_noalloc", _i, [C.POINTER(_vp), _i, _i, _i, _i, _i, _d, _d, _d, _d, _i, _i,
                                     C.POINTER(BgkDiag), _vp]),
    ("bgk_debug_stall_next_step", _i, [_vp]),
    ("bgk_strerror", C.c_char_p, [_i]),
    ("bgk_last_error", C.c_char_p, []),
    ("bgk_version", C.c_char_p, []),
]

_lib = None


class BgkError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {msg} (code {code})")
        self.code = code


def load(path: str | None = None):
    """Load libbgk3d.so (in-tree). Raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} is missing: build the CUDA library first (python -m bgk3d_hit_b200.build)")
    lib = C.CDLL(p)
    for name, res, args in PROTOTYPES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(rc: int, where: str, ok=(BGK_OK,)):
    if rc not in ok:
        lib = load()
        raise BgkError(rc, where, lib.bgk_last_error().decode() or lib.bgk_strerror(rc).decode())
    return rc
