"""bgk_diagnostics_noalloc: diagnostics for callers that cannot allocate.

Some callers cannot let the library call cudaMalloc once their time loop runs
(their device memory all belongs to another runtime, such as an OpenACC data
region, or to their own pool; cudaMalloc can fail on a full device and
synchronises it). This entry point reduces caller-owned device populations
with only a fixed file-scope device scratch array. Checked here:

- against the CPU oracle's diagno / dissipation / strain-rate sums on the same
  populations, and against the context entry point (bgk_diagnostic), within
  the diagnostics tolerance of the other GPU tests (1e-12 relative, 1e-15
  absolute), on calls in a row: each call sees the previous call's leftovers
  in the shared scratch and must not be affected by them;
- with caller rows padded (pitch_x > lx, the pad filled with NaN, which
  would poison every sum it reached) on a non-default stream;
- with no library context alive, device free memory is the same before and
  after a call (after one warm-up call that loads the kernels).

Enstrophy is not part of this entry point (it needs a velocity-field buffer).
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["rho_mean", "ux_mean", "uy_mean", "uz_mean", "ke_mean", "t", "tke_norm", "diss", "tke", "eps_strain"]
FORMS = {"fp64": "f64", "fp32": "f32", "fp16": "f16"}
F16_SCALE = 2.0 ** 16
SVISC, U0 = 0.005, 0.03


def _device_copy(pops, pitch_x=None, pad_value=np.nan):
    """The caller's own device copy of the populations (the caller allocates),
    rows optionally padded to pitch_x with pad_value."""
    import torch

    pops = np.ascontiguousarray(pops)
    nz, ny, nx = pops.shape[1:]
    px = pitch_x or nx
    host = np.full((19, nz, ny, px), pad_value, dtype=pops.dtype)
    host[..., :nx] = pops
    raw = host.view(np.uint8).reshape(-1)
    return torch.from_numpy(raw.copy()).cuda(), px


def _noalloc(bgk, dev, shape, pitch_x, precision, omega, mode, itime, stream=None):
    lib = bgk.load()
    nx, ny, nz = shape
    per = dev.numel() // 19
    ptrs = (C.c_void_p * 19)(*[dev.data_ptr() + q * per for q in range(19)])
    d = bgk._abi.BgkDiag()
    rc = lib.bgk_diagnostics_noalloc(ptrs, nx, ny, nz, pitch_x, bgk._abi.PRECISIONS[precision], SVISC, omega, U0,
                                     F16_SCALE if precision == "fp16" else 0.0, bgk._abi.MODES[mode], itime,
                                     C.byref(d), stream)
    assert rc == 0, lib.bgk_last_error()
    return d.as_dict()


def _oracle_states(O, shape, precision, steps):
    """Populations of a 3-component HIT field stepped by the oracle, with the
    oracle's own diagnostics of each state."""
    from bgk3d_hit_b200.hit import hit_velocity

    nx, ny, nz = shape
    u, v, w = hit_velocity((nz, ny, nx), k0=3, u_rms=U0, seed=77)
    orc = O.OracleLattice(nx, ny, nz, form=FORMS[precision], scale=F16_SCALE)
    orc.init_velocity(u, v, w, 1.0)
    out, it = [], 0
    for s in steps:
        while it < s:
            orc.step(SVISC, periodic=True)
            it += 1
        out.append((it, orc.get_pops(), orc.diagno(False), orc.diagno(True),
                    orc.dissipation(SVISC, U0, it, False), orc.extras(SVISC)))
    orc.close()
    return out


def _zj_last(pops, precision):
    """zj of the box's last cell (i = l, j = m, k = n) in the storage form's
    arithmetic, summed in the reference's order (SRC/diagno.F90:100-104)."""
    t = np.float64 if precision == "fp64" else np.float32
    x = pops[:, -1, -1, -1].astype(t)
    if precision == "fp16":
        x = x * np.float32(1.0 / F16_SCALE)
    rho = x[0]
    for q in range(1, 19):
        rho = t(rho + x[q])
    rho = t(rho + t(1))
    s = x[3]
    for q in (5, 6, 12, 17):
        s = t(s + x[q])
    for q in (1, 8, 10, 14, 15):
        s = t(s - x[q])
    return float(t(s * t(t(1) / rho)))


def _compare_oracle(got, itime, dg_c, zj_last, ds, ex, mode, ncell):
    """Faithful mode keeps the reference's ztot = ytot + zj (SRC/diagno.F90:110)
    but sums in compensated FP64 like corrected mode: uz_mean is the y mean
    plus the last cell's zj over the cell count (the oracle's faithful record
    instead runs single-precision sums in the FP32/FP16 forms)."""
    dg = np.array(dg_c)
    if mode == "faithful":
        dg[3] = dg_c[2] + zj_last / ncell
    np.testing.assert_allclose([got[f] for f in FIELDS[:5]], dg, rtol=1e-12, atol=1e-15)
    assert got["t"] == ds[0]
    np.testing.assert_allclose([got["tke_norm"], got["diss"], got["tke"]], ds[1:], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(got["eps_strain"], ex[1], rtol=1e-12, atol=1e-18)
    assert got["nonfinite"] == 0 and got["itime"] == itime


def _compare(got, ref):
    for f in FIELDS:
        assert got[f] == pytest.approx(ref[f], rel=1e-12, abs=1e-15), f
    assert got["nonfinite"] == ref["nonfinite"] == 0
    assert got["itime"] == ref["itime"]


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("mode", ["corrected", "faithful"])
def test_noalloc_matches_oracle_and_context_entry_point(bgk, oracle_mod, precision, mode):
    import torch

    shape = (24, 20, 16)
    omega = oracle_mod.omega(SVISC, FORMS[precision])
    states = _oracle_states(oracle_mod, shape, precision, (5, 12))
    devs = [_device_copy(s[1])[0] for s in states]
    torch.cuda.synchronize()
    # calls in a row on different states, then the first state again
    n = shape[0] * shape[1] * shape[2]
    for k in (0, 1, 0):
        it, pops, dg_c, dg_f, ds, ex = states[k]
        if mode == "faithful" and precision == "fp64":  # single rounding order: the oracle's own record
            np.testing.assert_allclose(dg_f[3], dg_c[2] + _zj_last(pops, precision) / n, rtol=1e-12, atol=1e-15)
        _compare_oracle(_noalloc(bgk, devs[k], shape, shape[0], precision, omega, mode, it), it, dg_c,
                        _zj_last(pops, precision), ds, ex, mode, n)
    # the context entry point on the same populations
    box = bgk.BGK3D(*shape, svisc=SVISC, u0=U0, precision=precision, icheck=1, mode=mode,
                    fp16_scale=F16_SCALE if precision == "fp16" else 0.0)
    try:
        for k in (1, 0):
            it, pops = states[k][:2]
            box.set_populations(pops)
            ref = box.diagnostic(it)
            _compare(_noalloc(bgk, devs[k], shape, shape[0], precision, omega, mode, it), ref)
    finally:
        box.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
def test_noalloc_padded_rows_on_a_caller_stream(bgk, oracle_mod, precision):
    """Rows padded by 3 (and by 32) elements of NaN: a row pitch handled wrong
    would read the pad and turn every sum non-finite, or shift the cells."""
    import torch

    shape = (21, 10, 9)
    omega = oracle_mod.omega(SVISC, FORMS[precision])
    (it, pops, dg_c, dg_f, ds, ex), = _oracle_states(oracle_mod, shape, precision, (3,))
    stream = torch.cuda.Stream()
    for pad in (3, 32):
        dev, px = _device_copy(pops, pitch_x=shape[0] + pad)
        stream.wait_stream(torch.cuda.current_stream())
        for _ in range(2):
            got = _noalloc(bgk, dev, shape, px, precision, omega, "corrected", it, stream=C.c_void_p(stream.cuda_stream))
            _compare_oracle(got, it, dg_c, 0.0, ds, ex, "corrected", 1)


def test_noalloc_allocates_no_device_memory(bgk, oracle_mod):
    """No library context is alive; one warm-up call loads the kernels (and
    the scratch array with them); later calls leave the device's free memory
    unchanged (cudaMemGetInfo, which sees any new device allocation of this
    process at the driver's page granularity)."""
    import gc

    import torch

    gc.collect()
    shape = (64, 32, 24)
    omega = oracle_mod.omega(SVISC, "f64")
    (it, pops, dg_c, dg_f, ds, ex), = _oracle_states(oracle_mod, shape, "fp64", (2,))
    dev, px = _device_copy(pops)
    torch.cuda.synchronize()
    _noalloc(bgk, dev, shape, px, "fp64", omega, "corrected", it)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        got = _noalloc(bgk, dev, shape, px, "fp64", omega, "corrected", it)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0
    _compare_oracle(got, it, dg_c, 0.0, ds, ex, "corrected", 1)


def test_noalloc_reports_nonfinite_with_a_message(bgk, oracle_mod):
    import torch

    shape = (8, 6, 5)
    (it, pops, *_), = _oracle_states(oracle_mod, shape, "fp64", (1,))
    pops = pops.copy()
    pops[3, 2, 1, 4] = np.nan
    dev, px = _device_copy(pops)
    torch.cuda.synchronize()
    lib = bgk.load()
    ptrs = (C.c_void_p * 19)(*[dev.data_ptr() + q * (dev.numel() // 19) for q in range(19)])
    d = bgk._abi.BgkDiag()
    rc = lib.bgk_diagnostics_noalloc(ptrs, *shape, px, 0, SVISC, 1.9, U0, 0.0, 0, it, C.byref(d), None)
    assert rc == bgk._abi.BGK_ERR_NONFINITE
    assert d.nonfinite == 1
    assert b"1 cells with non-finite" in lib.bgk_last_error()


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
