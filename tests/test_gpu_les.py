"""GPU tests of the LES (Smagorinsky) collision (params.les_cs > 0), the
reference's -DLES block of SRC/col_MC.F90:221-309, through the C-ABI.

Tolerance: bit-exact against the oracle in all three forms and both schemes
(the kernels round every operation, square roots included, as the oracle
does), with the FP16 four-cells-per-thread and FP32 two-cells-per-thread
kernels where a box fits them (rows inside a warp, one and several warps per
row); in FP16 kernel choices 2/8 fall back to the one cell per thread kernels
and give the same bits."""
import numpy as np
import pytest

from test_gpu_parity import F16_SCALE, FORMS, same_bits

pytestmark = pytest.mark.gpu

CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], float)


def _pair(bgk, O, shape, form, scheme, cs, svisc, init, kernel=0):
    nx, ny, nz = shape
    orc = O.OracleLattice(nx, ny, nz, form=FORMS[form], scale=F16_SCALE)
    if init == "tgv":
        orc.init_tgv(0.05)
    else:
        from bgk3d_hit_b200.hit import hit_velocity

        orc.init_velocity(*hit_velocity(nx, 2, 0.06, 11))
    orc.set_les(cs)
    box = bgk.BGK3D(nx, ny, nz, svisc=svisc, u0=0.05, precision=form, scheme=scheme,
                    fp16_scale=F16_SCALE if form == "fp16" else 0.0, les_cs=cs, kernel=kernel)
    box.set_populations(orc.get_pops())
    return orc, box


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
@pytest.mark.parametrize("case", [("tgv", (33, 20, 7), 0.17), ("hit", (16, 16, 16), 0.17),
                                  ("hit", (16, 16, 16), 1.0), ("tgv", (128, 8, 6), 0.17), ("tgv", (256, 4, 4), 1.0)])
def test_les_bitexact_vs_oracle(bgk, oracle_mod, form, scheme, case):
    init, shape, cs = case
    orc, box = _pair(bgk, oracle_mod, shape, form, scheme, cs, 1e-4, init)
    for it in range(1, 8):
        orc.step(1e-4, periodic=True)
        box.col_MC(it)
        if it in (1, 2, 7):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("kernel", [0, 2])
@pytest.mark.parametrize("case", [("tgv", (33, 20, 7), 0.17), ("hit", (16, 16, 16), 1.0), ("tgv", (128, 8, 6), 0.17),
                                  ("tgv", (512, 4, 3), 1.0)])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
def test_les_fp32_kernels_bitexact(bgk, oracle_mod, kernel, case, scheme):
    """The FP32 Smagorinsky steps with two cells per thread (and their
    fallback where a box does not fit) give the oracle's bits."""
    init, shape, cs = case
    orc, box = _pair(bgk, oracle_mod, shape, "fp32", scheme, cs, 1e-4, init, kernel=kernel)
    for it in range(1, 8):
        orc.step(1e-4, periodic=True)
        box.col_MC(it)
        if it in (1, 2, 7):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("kernel", [2, 4, 8])
def test_les_kernel_choices_fall_back_bitexact(bgk, oracle_mod, kernel):
    orc, box = _pair(bgk, oracle_mod, (32, 16, 8), "fp16", "two_lattice", 0.17, 1e-4, "tgv", kernel=kernel)
    for it in range(1, 5):
        orc.step(1e-4, periodic=True)
        box.col_MC(it)
    assert same_bits(box.populations(), orc.get_pops())
    box.close()


def test_les_zero_constant_is_the_bgk_path(bgk):
    a = bgk.BGK3D(16, svisc=0.01, les_cs=0.0)
    b = bgk.BGK3D(16, svisc=0.01)
    for box in (a, b):
        box.init()
        box.run(5)
    assert same_bits(a.populations(), b.populations())
    a.close()
    b.close()


def test_les_stabilises_an_under_resolved_box(bgk):
    """HIT at tau = 0.5002 on 32^3 (u_rms 0.08): BGK leaves the physical
    range within 500 steps, the Smagorinsky closure (cteS = 0.17) decays."""
    from bgk3d_hit_b200.hit import hit_velocity

    n = 32
    u = hit_velocity(n, 4, 0.08, 1234)
    out = {}
    for cs in (0.0, 0.17):
        box = bgk.BGK3D(n, svisc=0.0002 / 3, u0=0.08, les_cs=cs)
        box.init_velocity(*u)
        box.run(500)
        d = box.deviations()
        with np.errstate(all="ignore"):
            ux = np.tensordot(CX, d, 1) / (d.sum(0) + 1.0)
            out[cs] = float(np.sqrt(np.mean(ux * ux)))
        box.close()
    assert not (out[0.0] < 1.0)
    assert np.isfinite(out[0.17]) and out[0.17] < 0.03


def test_les_rejected_where_unsupported(bgk):
    import ctypes as C

    lib = bgk.load()
    box = bgk.BGK3D(8, les_cs=0.17, kernel=8)
    assert lib.bgk_debug_stall_next_step(box._h) == bgk._abi.BGK_ERR_INVALID
    u = [np.zeros(512)] * 3
    dp = C.POINTER(C.c_double)
    ptr = [a.ctypes.data_as(dp) for a in u]
    loss = C.c_double()
    rc = lib.bgk_adjoint(box._h, *ptr, *ptr, 4, 2, C.byref(loss), None, None)
    assert rc == bgk._abi.BGK_ERR_INVALID
    box.close()
