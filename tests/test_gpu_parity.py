"""GPU parity of the CUDA path against the oracle, through the C-ABI.

Tolerances (written per test):
- stream-collide from identical input populations: bit-exact in all three
  forms (the kernels round every operation as the oracle does);
- Taylor-Green init: CUDA's sin/cos versus the C library's, |diff| <= 1e-14
  (FP64) or 4e-6 (FP32) times the largest deviation;
- diagnostics: compensated FP64 sums in a different order than the oracle's,
  <= 1e-12 relative (or 1e-15 absolute for quantities that vanish).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORMS = {"fp64": "f64", "fp32": "f32", "fp16": "f16"}
F16_SCALE = 2.0 ** 16


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def make_pair(bgk, O, shape, form, scheme="two_lattice", svisc=0.01, faithful=True, **kw):
    nx, ny, nz = shape
    orc = O.OracleLattice(nx, ny, nz, form=FORMS[form], scale=F16_SCALE)
    orc.init_tgv(0.05, faithful=faithful)
    box = bgk.BGK3D(nx, ny, nz, svisc=svisc, u0=0.05, precision=form, scheme=scheme,
                    fp16_scale=F16_SCALE if form == "fp16" else 0.0, **kw)
    box.set_populations(orc.get_pops())
    return orc, box


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("shape", [(5, 7, 9), (17, 17, 17), (64, 64, 64), (33, 20, 7)])
def test_two_lattice_bitexact_vs_oracle(bgk, oracle_mod, form, shape):
    orc, box = make_pair(bgk, oracle_mod, shape, form)
    assert same_bits(box.populations(), orc.get_pops())
    orc.step(0.01, periodic=True)
    box.boundaries(1)
    box.col_MC(1)
    assert same_bits(box.populations(), orc.get_pops()), "after 1 step"
    for it in range(2, 11):
        orc.step(0.01, periodic=True)
        box.boundaries(it)
        box.col_MC(it)
    assert same_bits(box.populations(), orc.get_pops()), "after 10 steps"
    box.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
def test_hit64_bitexact_vs_oracle(bgk, oracle_mod, form, scheme):
    """64^3 decaying-HIT initial condition (k0 = 4, u_rms = 0.03), 1 and 10
    steps, every form and scheme: the oracle's bits."""
    from bgk3d_hit_b200.hit import hit_velocity

    n = 64
    u = hit_velocity(n, 4, 0.03, 1234)
    orc = oracle_mod.OracleLattice(n, n, n, form=FORMS[form], scale=F16_SCALE)
    orc.init_velocity(*u)
    box = bgk.BGK3D(n, svisc=0.005 / 3, precision=form, scheme=scheme,
                    fp16_scale=F16_SCALE if form == "fp16" else 0.0)
    box.init_velocity(*u)
    for it in range(1, 11):
        orc.step(0.005 / 3, periodic=True)
        box.col_MC(it)
        if it in (1, 10):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("kernel", [1, 2, 4])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 16, 8), (8, 8, 8), (256, 4, 4), (128, 6, 5), (24, 8, 6)])
def test_fp16_kernel_variants_bitexact(bgk, oracle_mod, kernel, shape):
    """The one-, two- and four-cells-per-thread FP16 kernels (warp-shuffle
    x-shifts, cross-warp loads when a row spans several warps, fallback where a
    box does not fit) give the oracle's bits."""
    orc, box = make_pair(bgk, oracle_mod, shape, "fp16", kernel=kernel)
    for it in range(1, 6):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
    assert same_bits(box.populations(), orc.get_pops())
    box.close()


@pytest.mark.parametrize("kernel", [0, 1, 2])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 16, 8), (8, 8, 8), (256, 4, 4), (128, 6, 5), (24, 8, 6),
                                   (1024, 4, 4), (64, 3, 2)])
def test_fp32_two_lattice_kernel_variants_bitexact(bgk, oracle_mod, kernel, shape):
    """The two-cells-per-thread FP32 two-lattice kernel (warp-shuffle
    x-shifts, cross-warp loads when a row spans several warps, fallback where a
    box does not fit) gives the oracle's bits."""
    orc, box = make_pair(bgk, oracle_mod, shape, "fp32", kernel=kernel)
    for it in range(1, 6):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
        if it in (1, 5):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("kernel", [0, 1, 2])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 16, 8), (8, 8, 8), (256, 4, 4), (128, 6, 5), (24, 8, 6),
                                   (512, 2, 3), (1024, 4, 4), (64, 3, 2), (2048, 2, 2)])
def test_fp32_aa_kernel_variants_bitexact(bgk, oracle_mod, kernel, shape):
    """The two-cells-per-thread FP32 AA kernels (rows inside a warp, one,
    two and four warps per row, rows over two and four blocks, blocks with
    idle warps, fallback where a box does not fit) give the oracle's bits
    over steps of both parities."""
    orc, box = make_pair(bgk, oracle_mod, shape, "fp32", scheme="aa", kernel=kernel)
    for it in range(1, 6):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
        if it in (1, 2, 5):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("kernel", [0, 1, 4])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 16, 8), (8, 8, 8), (256, 4, 4), (128, 6, 5), (24, 8, 6),
                                   (512, 2, 3)])
def test_fp16_aa_kernel_variants_bitexact(bgk, oracle_mod, kernel, shape):
    """The four-cells-per-thread FP16 AA kernels (x-crossing values moved
    between lanes on loads and stores; rows inside a warp, one warp and
    several warps per row; fallback where a box does not fit) give the
    oracle's bits over steps of both parities."""
    orc, box = make_pair(bgk, oracle_mod, shape, "fp16", scheme="aa", kernel=kernel)
    for it in range(1, 6):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
        if it in (1, 2, 5):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("shape", [(64, 32, 5), (256, 8, 6), (1024, 4, 3), (2048, 2, 3), (16, 64, 3),
                                   (8, 128, 3), (128, 16, 8)])
def test_fp16_aa_eight_cells_odd_step_bitexact(bgk, oracle_mod, shape):
    """The automatic FP16 AA odd step with eight cells per thread (16-byte
    chunks; rows of one lane, inside a warp, one warp, four warps in one block,
    and eight warps over two blocks, whose block-boundary lanes store partial
    chunks) gives the oracle's bits over steps of both parities, as does the
    four-cells kernel it replaces (kernel = 4)."""
    for kernel in (0, 4):
        orc, box = make_pair(bgk, oracle_mod, shape, "fp16", scheme="aa", kernel=kernel)
        for it in range(1, 6):
            orc.step(0.01, periodic=True)
            box.col_MC(it)
            if it in (1, 2, 5):
                assert same_bits(box.populations(), orc.get_pops()), f"kernel {kernel}, after {it} steps"
        box.close()


@pytest.mark.parametrize("les_cs", [0.0, 0.17])
@pytest.mark.parametrize("shape", [(64, 32, 5), (256, 8, 6), (1024, 4, 3), (2048, 2, 3), (16, 64, 3),
                                   (8, 128, 3), (4, 256, 2), (128, 16, 8)])
def test_fp32_aa_four_cells_odd_step_bitexact(bgk, oracle_mod, shape, les_cs):
    """The automatic FP32 AA odd step with four cells per thread (16-byte
    chunks; rows of one lane, inside a warp, one and two warps, and eight
    warps over two blocks with partial chunks at the block boundary), with
    the BGK and the Smagorinsky collision, gives the oracle's bits over steps
    of both parities, as does the two-cells kernel (kernel = 2)."""
    for kernel in (0, 2):
        orc, box = make_pair(bgk, oracle_mod, shape, "fp32", scheme="aa", kernel=kernel, les_cs=les_cs)
        orc.set_les(les_cs)
        for it in range(1, 6):
            orc.step(0.01, periodic=True)
            box.col_MC(it)
            if it in (1, 2, 5):
                assert same_bits(box.populations(), orc.get_pops()), f"kernel {kernel}, after {it} steps"
        box.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
@pytest.mark.parametrize("shape", [(5, 7, 9), (64, 16, 8), (33, 20, 7), (256, 3, 2)])
def test_row_pipeline_kernel_bitexact(bgk, oracle_mod, form, scheme, shape):
    """The TMA row-pipelined kernel (kernel 8) gives the oracle's bits in both
    schemes, over steps of both AA parities."""
    orc, box = make_pair(bgk, oracle_mod, shape, form, scheme=scheme, kernel=8)
    for it in range(1, 8):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
        if it in (1, 2, 7):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


def test_row_pipeline_bounded_wait_reports_and_recovers(bgk, oracle_mod):
    """A wait that runs out (injected: a barrier nothing arms) abandons the
    step, is reported at the next synchronisation, and the context recovers
    after a new initialisation. No fault is involved."""
    B = bgk
    orc, box = make_pair(bgk, oracle_mod, (64, 16, 8), "fp64", kernel=8)
    lib = B.load()
    assert lib.bgk_debug_stall_next_step(box._h) == 0
    box.col_MC(1)
    with pytest.raises(B.BgkError) as e:
        box.synchronize()
    assert e.value.code == B._abi.BGK_ERR_CUDA and "gave up" in str(e.value)
    box.set_populations(orc.get_pops())
    orc.step(0.01, periodic=True)
    box.col_MC(1)
    box.synchronize()
    assert same_bits(box.populations(), orc.get_pops())
    box.close()
    plain = B.BGK3D(8, kernel=1)
    with pytest.raises(B.BgkError):
        B._abi.check(lib.bgk_debug_stall_next_step(plain._h), "stall")
    plain.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("shape", [(5, 7, 9), (32, 16, 8)])
def test_aa_pattern_bitexact_vs_oracle(bgk, oracle_mod, form, shape):
    orc, box = make_pair(bgk, oracle_mod, shape, form, scheme="aa")
    for it in range(1, 12):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
        if it in (1, 2, 7, 10, 11):
            assert same_bits(box.populations(), orc.get_pops()), f"after {it} steps"
    box.close()


@pytest.mark.parametrize("mode", ["faithful", "corrected"])
@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
def test_tgv_init_vs_oracle(bgk, oracle_mod, mode, form, scheme):
    shape = (12, 10, 14)
    orc = oracle_mod.OracleLattice(*shape, form=FORMS[form])
    orc.init_tgv(0.05, faithful=(mode == "faithful"))
    box = bgk.BGK3D(*shape, svisc=0.01, u0=0.05, precision=form, scheme=scheme, mode=mode)
    box.init()
    g, r = box.deviations(), orc.get_dev()
    tol = (1e-14 if form == "fp64" else 4e-6) * np.abs(r).max()
    assert np.abs(g - r).max() <= tol
    box.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
def test_velocity_init_bitexact(bgk, oracle_mod, form, scheme):
    shape = (9, 8, 7)
    n = 9 * 8 * 7
    rng = np.random.default_rng(5)
    u, v, w = (rng.uniform(-0.04, 0.04, n) for _ in range(3))
    orc = oracle_mod.OracleLattice(*shape, form=FORMS[form], scale=F16_SCALE)
    orc.init_velocity(u, v, w, 1.0)
    box = bgk.BGK3D(*shape, precision=form, scheme=scheme, fp16_scale=F16_SCALE if form == "fp16" else 0.0)
    box.init_velocity(u, v, w, 1.0)
    assert same_bits(box.populations(), orc.get_pops())
    box.close()


def test_fp16_auto_scale_is_power_of_two(bgk):
    box = bgk.BGK3D(16, precision="fp16", u0=0.05)
    box.init()
    s = box.scale
    assert s > 1 and np.log2(s) == int(np.log2(s))
    d = np.abs(box.deviations()).max()
    assert 65504 / 8 < d * s <= 65504 / 4
    box.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
@pytest.mark.parametrize("nsteps", [0, 1, 4])
def test_diagnostics_vs_oracle(bgk, oracle_mod, form, scheme, nsteps):
    shape = (16, 12, 10)
    orc, box = make_pair(bgk, oracle_mod, shape, form, scheme=scheme, icheck=1)
    for it in range(1, nsteps + 1):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
    itime = max(nsteps, 1)
    d = box.diagnostic(itime)
    dg = orc.diagno(False)
    ds = orc.dissipation(0.01, 0.05, itime, False)
    ex = orc.extras(0.01)
    got = [d["rho_mean"], d["ux_mean"], d["uy_mean"], d["uz_mean"], d["ke_mean"]]
    np.testing.assert_allclose(got, dg, rtol=1e-12, atol=1e-15)
    assert d["t"] == ds[0]
    np.testing.assert_allclose([d["tke_norm"], d["diss"], d["tke"]], ds[1:], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose([d["enstrophy"], d["eps_strain"]], ex[:2], rtol=1e-12, atol=1e-18)
    assert d["nonfinite"] == 0
    box.close()


def test_faithful_diagno_ztot(bgk, oracle_mod):
    orc, box = make_pair(bgk, oracle_mod, (10, 9, 8), "fp64", mode="faithful", icheck=1)
    for it in range(1, 4):
        orc.step(0.01, periodic=True)
        box.col_MC(it)
    got = box.diagno(3)
    ref = orc.diagno(True)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)
    box.close()


def test_diagnostic_gating_and_ungated_calls(bgk):
    box = bgk.BGK3D(8, icheck=5)
    box.init()
    assert box.diagnostic(3) is None
    assert box.diagnostic(5) is not None
    d5, s5 = box.diagno(5), box.dissipation(5)
    assert d5.shape == (5,) and s5.shape == (4,)
    box.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
def test_velocity_and_spectrum_parseval(bgk, oracle_mod, form):
    from bgk3d_hit_b200.hit import hit_velocity

    u, v, w = hit_velocity(24, k0=3, u_rms=0.03, seed=9)
    box = bgk.BGK3D(24, precision=form)
    box.init_velocity(u, v, w)
    gu, gv, gw = box.velocity()
    tol = 1e-15 if form == "fp64" else (5e-8 if form == "fp32" else 5e-5)
    assert np.abs(gu - u).max() < tol and np.abs(gv - v).max() < tol and np.abs(gw - w).max() < tol
    ek = box.spectrum(40)
    ke = 0.5 * (gu * gu + gv * gv + gw * gw).mean()
    assert ek.sum() == pytest.approx(ke, rel=1e-9 if form == "fp64" else 1e-5)
    assert abs(int(np.argmax(ek)) - 3) <= 1
    box.close()


def test_shift3_matches_numpy_roll(bgk):
    import torch

    for dt, es in ((torch.float64, 8), (torch.float32, 4), (torch.float16, 2)):
        nx, ny, nz = 13, 6, 5
        ins = [torch.randn(nz, ny, nx, dtype=torch.float32, device="cuda").to(dt) for _ in range(3)]
        for rev in (0, 1):
            outs = [torch.empty_like(t) for t in ins]
            lib = bgk.load()
            rc = lib.bgk_shift3(*[t.data_ptr() for t in ins], *[t.data_ptr() for t in outs], nx, ny, nz, es, rev,
                                None)
            assert rc == 0
            torch.cuda.synchronize()
            s = -1 if rev else 1
            exp = [torch.roll(ins[0], s, 2), torch.roll(ins[1], s, 1), torch.roll(ins[2], s, 0)]
            for a, b in zip(outs, exp):
                assert torch.equal(a, b)


def test_pure_streaming_delta_gpu(bgk):
    """omega = 0 turns the step into pure streaming: each delta moves to
    (x + c_q) mod L (the reference's wrap, SRC/bcond.comm.step3.F90)."""
    cx = [1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0]
    cy = [-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0]
    cz = [0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0]
    l, m, n = 5, 7, 9
    for scheme in ("two_lattice", "aa"):
        box = bgk.BGK3D(l, m, n, omega=0.0, scheme=scheme)
        a = np.zeros((19, n, m, l))
        for q in range(18):
            a[q, (2 * q) % n, q % m, (3 * q) % l] = 1.0 + q
        box.set_populations(a)
        box.col_MC(1)
        b = box.populations()
        exp = np.zeros_like(a)
        for q in range(18):
            exp[q, (2 * q + cz[q]) % n, (q + cy[q]) % m, (3 * q + cx[q]) % l] = 1.0 + q
        assert np.array_equal(b, exp), scheme
        box.close()


def test_conservation_fp64_long_run(bgk):
    from bgk3d_hit_b200.hit import hit_velocity

    u, v, w = hit_velocity(32, k0=4, u_rms=0.03, seed=1234)
    box = bgk.BGK3D(32, svisc=0.005 / 3, precision="fp64", icheck=1)
    box.init_velocity(u, v, w)
    d0 = box.deviations()
    box.run(200)
    d1 = box.deviations()
    assert abs(d1.sum() - d0.sum()) < 1e-12
    for c in ([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0],):
        cc = np.array(c, float)
        assert abs(np.tensordot(cc, d1, 1).sum() - np.tensordot(cc, d0, 1).sum()) < 1e-12
    box.close()


def test_tgv_viscous_decay_gpu(bgk):
    """Known answer at vanishing Reynolds number: rate 2 nu |k|^2 within 1%."""
    L0, nu, steps = 32, 0.02, 300
    box = bgk.BGK3D(L0, svisc=nu, u0=1e-4, icheck=1)
    box.init()
    box.col_MC(1)
    ke1 = box.diagno(1)[4]
    box.run(steps)
    ke = box.diagno(steps + 1)[4]
    k2 = 3 * (2 * np.pi / L0) ** 2
    assert np.log(ke / ke1) / (-2 * nu * k2 * steps) == pytest.approx(1.0, abs=1e-2)
    box.close()


def test_error_paths(bgk):
    B = bgk
    box = B.BGK3D(8)
    with pytest.raises(B.BgkError) as e:
        box.col_MC(1)
    assert e.value.code == B._abi.BGK_ERR_STATE
    box.init()
    pops = box.populations()
    pops[3, 1, 2, 3] = np.nan
    box.set_populations(pops)
    with pytest.raises(B.BgkError) as e:
        box.diagnostic(10)
    assert e.value.code == B._abi.BGK_ERR_NONFINITE
    box.close()
    with pytest.raises(B.BgkError) as e:
        B.BGK3D(8, device=99)
    assert e.value.code == B._abi.BGK_ERR_INVALID


def test_run_loop_writes_reference_files(bgk, tmp_path):
    from bgk3d_hit_b200 import run_loop

    box = bgk.BGK3D(16, svisc=0.01, u0=0.05, icheck=5, mode="faithful")
    box.init()
    recs = run_loop(box, 20, str(tmp_path))
    assert [r["itime"] for r in recs] == [5, 10, 15, 20]
    lines = (tmp_path / "diagno.dat").read_text().splitlines()
    assert len(lines) == 4 and len(lines[0].split()) == 6
    assert abs(float(lines[0].split()[4]) - 1.0) < 1e-6
    assert len((tmp_path / "dissipation.dat").read_text().splitlines()[0].split()) == 4
    box.close()


@pytest.mark.parametrize("mode", ["corrected", "faithful"])
def test_tgv64_full_run_energy_and_dissipation_curves_vs_oracle(bgk, oracle_mod, mode):
    """Config C1 as a whole run: Taylor-Green 64^3, FP64, tau = 0.53
    (svisc 0.01), U0 = 0.05, 500 steps, diagnostics every 10 steps. The GPU's
    E(t) and dissipation curves match the oracle's to 1e-9 relative at every
    record (the populations stay bit-exact, so the difference is only the
    order of the compensated sums), and the populations still match bit for
    bit at the end. Faithful mode: the oracle runs the reference's loop body
    (step3 ghost fill + col_MC) and its dissipation reads the stale ghosts the
    reference reads."""
    n, svisc, u0 = 64, 0.01, 0.05
    faithful = mode == "faithful"
    orc = oracle_mod.OracleLattice(n, n, n)
    orc.init_tgv(u0, faithful=True)
    box = bgk.BGK3D(n, svisc=svisc, u0=u0, icheck=10, mode=mode)
    box.set_populations(orc.get_pops())
    worst = 0.0
    for it in range(1, 501):
        orc.step(svisc, periodic=not faithful)
        box.col_MC(it)
        d = box.diagnostic(it)
        if d is None:
            continue
        dg = orc.diagno(False)
        ds = orc.dissipation(svisc, u0, it, 2 if faithful else 0)
        for got, ref in ((d["ke_mean"], dg[4]), (d["tke_norm"], ds[1]), (d["diss"], ds[2]), (d["rho_mean"], dg[0])):
            worst = max(worst, abs(got - ref) / abs(ref))
    assert worst <= 1e-9, worst
    assert same_bits(box.populations(), orc.get_pops())
    box.close()
