"""The FP16 form's collision against the reference's FP64 col_MC.

The FP16 storage form has its own collision formulation (scaled stored values,
dr kept apart from 1, opposite directions in pairs with fused multiply-adds;
the oracle's fast16_cell, which the CUDA kernels follow operation for
operation). The FP16 kernels are bit-exact against that restatement on the
GPU; this file pins the restatement itself to the reference algorithm: the
oracle's FP64 col_MC (SRC/col_MC.F90:133-351) on the same inputs.

Set-up: random cells with velocities up to 0.05 / 0.15 / 0.3, densities
1 +- 0.05 and non-equilibrium parts of 1e-3 to 3e-2 relative; stored in
binary16 as y = scale*(f - w) with the library's scale rule
2^floor(log2(65504 / (4 max|f - w|))); the FP64 lattice gets the same values
decoded exactly (y / scale). One step of each with periodic pulls (streaming
is an exact permutation, so every cell sees identical inputs).

Bound per output value, in scaled units:
    |y16' - scale*f64'| <= ulp16(scale*f64') / 2 + eps * max|y|
The first term is the binary16 output rounding. The second covers the FP32
arithmetic of the form (and omega rounded to FP32): eps = 2e-7 for BGK, 1e-6
for the Smagorinsky closure (measured worst cases 4.5e-8 and 2.0e-7 of
max|y| over these sets).
"""
import numpy as np
import pytest

CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], float)
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0], float)
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], float)
_N1 = np.abs(CX) + np.abs(CY) + np.abs(CZ)
W = np.where(_N1 == 2, 1 / 36, np.where(_N1 == 1, 1 / 18, 1 / 3))


def ulp16(x):
    """Spacing of binary16 numbers at |x| (subnormal spacing below 2^-14)."""
    e = np.floor(np.log2(np.maximum(np.abs(x), 2.0 ** -14)))
    return 2.0 ** (e - 10)


def random_cells(rng, shape, umax, noneq):
    nx, ny, nz = shape
    u = rng.uniform(-umax, umax, (3, nz, ny, nx))
    rho = 1 + rng.uniform(-0.05, 0.05, (nz, ny, nx))
    cu = CX[:, None, None, None] * u[0] + CY[:, None, None, None] * u[1] + CZ[:, None, None, None] * u[2]
    feq = W[:, None, None, None] * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (u * u).sum(0))
    f = feq * (1 + noneq * rng.standard_normal(feq.shape))
    dev = f - W[:, None, None, None]
    scale = 2.0 ** np.floor(np.log2(65504 / (4 * np.abs(dev).max())))
    y = (dev * scale).astype(np.float16)
    return y, y.astype(np.float64) / scale, scale


@pytest.mark.parametrize("les_cs", [0.0, 0.17])
@pytest.mark.parametrize("umax,noneq", [(0.05, 1e-3), (0.15, 1e-2), (0.3, 3e-2)])
@pytest.mark.parametrize("svisc", [0.01, 0.005 / 3, 1e-4])
def test_fp16_collision_matches_fp64_col_mc(oracle_mod, les_cs, umax, noneq, svisc):
    O = oracle_mod
    shape = (16, 12, 10)
    rng = np.random.default_rng(int(1e6 * umax) + int(1e9 * svisc) + int(100 * les_cs))
    y, d, scale = random_cells(rng, shape, umax, noneq)
    a = O.OracleLattice(*shape, "f64")
    h = O.OracleLattice(*shape, "f16", scale=scale)
    for L, p in ((a, d), (h, y)):
        L.set_les(les_cs)
        L.put_pops(p)
        L.step(svisc, periodic=True)
    ref = a.get_dev() * scale
    got = h.get_pops().astype(np.float64)
    a.close()
    h.close()
    eps = 1e-6 if les_cs > 0 else 2e-7
    bound = 0.5 * ulp16(ref) + eps * np.abs(y.astype(np.float64)).max()
    excess = np.abs(got - ref) - bound
    assert excess.max() <= 0, f"worst excess {excess.max():.3g} (scaled units)"
    # the output rounding dominates: nearly every value is correctly rounded
    assert np.mean(np.abs(got - ref) <= 0.5 * ulp16(ref) * (1 + 1e-6)) > 0.95


def test_fp16_collision_sees_the_relaxation(oracle_mod):
    """Guard against a vacuous bound: the FP64 step moves the values by many
    binary16 ulps, so a form that skipped the collision would fail above."""
    O = oracle_mod
    shape = (8, 6, 5)
    y, d, scale = random_cells(np.random.default_rng(3), shape, 0.15, 1e-2)
    a = O.OracleLattice(*shape, "f64")
    a.put_pops(d)
    a.step(0.01, periodic=True)
    moved = np.abs(a.get_dev() * scale - d * scale)
    a.close()
    assert np.median(moved / ulp16(d * scale)) > 10
