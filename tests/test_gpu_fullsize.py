"""Full-size boxes of the benchmarked configurations, checked through a
size-independent property: translation invariance.

A box of L^3 cells initialised with a 256^3 HIT field tiled (L/256)^3 times
must evolve as the exact tiling of the 256^3 box's run: every cell applies
the same arithmetic to the same inputs, so any indexing error that only large
boxes reach (32-bit offsets, the 1024-cell rows of the four-cells-per-thread
FP16 kernels, grid shapes, staging chunks) shows up as a difference. Checked
bit for bit on single-precision velocity slices (the VTK writer's j/rho) in
all three orientations at planes inside and across tile borders, after steps
of both AA parities; the diagnostics (sums over 64x or 8x more cells in
another order) agree to 1e-12 relative. The 256^3 tile itself is pinned to
the oracle by the other parity tests.

Boxes: the AA pattern at 1024^3 in FP16 (41 GB) and FP32 (82 GB) storage,
and FP64 two-lattice at 512^3 (40 GB).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILE = 256


def _slice(box, kind, index1, itime, tmp):
    getattr(box, {"xy": "vtk_xy_bin", "xz": "vtk_xz_bin", "yz": "vtk_yz_bin"}[kind])(itime, index1, str(tmp))
    raw = open(tmp / f"tec_{kind}.00000.{itime:08d}.vtk", "rb").read()
    pos = 0
    for _ in range(9):
        pos = raw.index(b"\n", pos) + 1
    return np.frombuffer(raw[pos:], dtype=">f4")


@pytest.mark.parametrize("L,form,scheme", [(1024, "fp16", "aa"), (1024, "fp32", "aa"), (512, "fp64", "two_lattice")])
def test_tiled_box_evolves_as_its_tile(bgk, tmp_path, L, form, scheme):
    import torch

    from bgk3d_hit_b200.hit import hit_velocity

    rep, n, steps = L // TILE, TILE, 6
    svisc = 0.002 / 3
    u = hit_velocity(n, 4, 0.03, 1234)
    small = bgk.BGK3D(n, svisc=svisc, u0=0.03, precision=form, scheme=scheme, icheck=steps)
    small.init_velocity(*u)
    big = bgk.BGK3D(L, svisc=svisc, u0=0.03, precision=form, scheme=scheme, icheck=steps,
                    fp16_scale=small.scale if form == "fp16" else 0.0)
    try:
        tiled = [torch.from_numpy(x).cuda().repeat(rep, rep, rep) for x in u]
        big.init_velocity_device(*tiled)
        del tiled
        torch.cuda.empty_cache()
        small.run(steps)
        big.run(steps)
        ds, db = small.diagnostic(steps), big.diagnostic(steps)
        for f in ("rho_mean", "ux_mean", "uy_mean", "uz_mean", "ke_mean", "tke_norm", "diss", "eps_strain"):
            want = ds[f] * (rep ** 3 if f == "diss" else 1)  # diss is a sum over the cells, the others means
            assert db[f] == pytest.approx(want, rel=1e-12, abs=1e-15), f
        for kind in ("xy", "xz", "yz"):
            for idx in (1, 2, n, n + 1, n + 37, L - 5, L):
                got = _slice(big, kind, idx, steps, tmp_path).reshape(L, L, 3)
                ref = _slice(small, kind, (idx - 1) % n + 1, steps, tmp_path).reshape(n, n, 3)
                assert np.array_equal(got, np.tile(ref, (rep, rep, 1))), (kind, idx)
    finally:
        big.close()
        small.close()
