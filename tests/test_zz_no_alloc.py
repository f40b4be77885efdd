"""bgk_diagnostics_noalloc: diagnostics for callers that cannot allocate.

Some callers cannot let the library call cudaMalloc once their time loop runs
(their device memory all belongs to another runtime or to their own pool, and
cudaMalloc can fail on a full device and synchronises it). This entry point
reduces caller-owned device populations with only a fixed file-scope device
scratch array. Here it must give the same diagnostics as the context entry
point (bgk_diagnostic) on the same populations, within the diagnostics
tolerance of the other GPU tests (1e-12 relative, 1e-15 absolute), on two
calls in a row: the second call sees the first call's leftovers in the shared
scratch and must not be affected by them. Enstrophy is not part of this entry
point (it needs a velocity-field buffer).

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["rho_mean", "ux_mean", "uy_mean", "uz_mean", "ke_mean", "t", "tke_norm", "diss", "tke", "eps_strain"]


def _device_copy(pops):
    """The caller's own device copy of the populations (the caller allocates)."""
    import torch

    raw = np.ascontiguousarray(pops).view(np.uint8)
    return torch.from_numpy(raw.copy()).cuda()


def _noalloc(bgk, dev, shape, precision, box, mode, itime):
    lib = bgk.load()
    nx, ny, nz = shape
    per = dev.numel() // 19
    ptrs = (C.c_void_p * 19)(*[dev.data_ptr() + q * per for q in range(19)])
    d = bgk._abi.BgkDiag()
    rc = lib.bgk_diagnostics_noalloc(ptrs, nx, ny, nz, nx, bgk._abi.PRECISIONS[precision], box.params.svisc,
                                     box.omega, box.params.u0, box.scale if precision == "fp16" else 0.0,
                                     bgk._abi.MODES[mode], itime, C.byref(d), None)
    assert rc == 0, lib.bgk_last_error()
    return d.as_dict()


def _compare(got, ref):
    for f in FIELDS:
        assert got[f] == pytest.approx(ref[f], rel=1e-12, abs=1e-15), f
    assert got["nonfinite"] == ref["nonfinite"] == 0
    assert got["itime"] == ref["itime"]


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("mode", ["corrected", "faithful"])
def test_noalloc_matches_context_entry_point(bgk, precision, mode):
    import torch

    from bgk3d_hit_b200.hit import hit_velocity

    shape = (24, 20, 16)
    u, v, w = hit_velocity(shape[::-1], k0=3, u_rms=0.03, seed=77)
    box = bgk.BGK3D(*shape, svisc=0.005, u0=0.03, precision=precision, icheck=1, mode=mode)
    box.init_velocity(u, v, w)
    box.run(5)
    ref5 = box.diagnostic(5)
    dev5 = _device_copy(box.populations())
    box.run(7)
    ref12 = box.diagnostic(12)
    dev12 = _device_copy(box.populations())
    torch.cuda.synchronize()
    # two calls in a row on different states, then the first state again
    _compare(_noalloc(bgk, dev5, shape, precision, box, mode, 5), ref5)
    _compare(_noalloc(bgk, dev12, shape, precision, box, mode, 12), ref12)
    _compare(_noalloc(bgk, dev5, shape, precision, box, mode, 5), ref5)
    box.close()


def test_noalloc_rejects_oversized_and_invalid_boxes(bgk):
    import torch

    lib = bgk.load()
    buf = torch.zeros(19 * 8, dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * 19)(*[buf.data_ptr() + 64 * q for q in range(19)])
    d = bgk._abi.BgkDiag()
    rc = lib.bgk_diagnostics_noalloc(ptrs, 2048, 1024, 1024, 2048, 0, 0.01, 1.9, 0.05, 0.0, 0, 1, C.byref(d), None)
    assert rc == bgk._abi.BGK_ERR_INVALID
    assert b"too large" in lib.bgk_last_error()
    rc = lib.bgk_diagnostics_noalloc(ptrs, 8, 1, 1, 4, 0, 0.01, 1.9, 0.05, 0.0, 0, 1, C.byref(d), None)
    assert rc == bgk._abi.BGK_ERR_INVALID
    rc = lib.bgk_diagnostics_noalloc(ptrs, 2, 2, 2, 2, 2, 0.01, 1.9, 0.05, 3.0, 0, 1, C.byref(d), None)
    assert rc == bgk._abi.BGK_ERR_INVALID
