"""GPU tests of the discrete adjoint (bgk_adjoint) and tangent-linear model
(bgk_tangent): no reference counterpart exists, so they are checked against
each other (dot-product test), against central finite differences of the
loss computed on the GPU and on the CPU oracle (whose forward step is
bit-exact with the GPU's), and for independence from the checkpoint interval.

Tolerances: dot-product test 1e-9 relative (FP64); finite differences with
h = 1e-6, 1e-6 relative (FP64), 2e-3 relative (FP32, h = 1e-3).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DP = C.POINTER(C.c_double)


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(DP)


def fields(n, seed, amp=0.03):
    from bgk3d_hit_b200.hit import hit_velocity

    return hit_velocity(n, k0=2, u_rms=amp, seed=seed)


def adjoint(box, u0, ut, T, K, grads=True):
    lib = box._lib
    n = box.ncell
    loss = C.c_double()
    gu = np.zeros(3 * n) if grads else None
    gt = C.c_double()
    rc = lib.bgk_adjoint(box._h, _p(u0[0]), _p(u0[1]), _p(u0[2]), _p(ut[0]), _p(ut[1]), _p(ut[2]), T, K,
                         C.byref(loss), gu.ctypes.data_as(DP) if grads else None, C.byref(gt) if grads else None)
    assert rc == 0, lib.bgk_last_error()
    return loss.value, gu, gt.value


def tangent(box, u0, du, dtau, ut, T):
    lib = box._lib
    loss, dl = C.c_double(), C.c_double()
    rc = lib.bgk_tangent(box._h, _p(u0[0]), _p(u0[1]), _p(u0[2]), _p(du[0]), _p(du[1]), _p(du[2]), dtau,
                         _p(ut[0]), _p(ut[1]), _p(ut[2]), T, C.byref(loss), C.byref(dl))
    assert rc == 0, lib.bgk_last_error()
    return loss.value, dl.value


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_adjoint_matches_tangent_linear(bgk, precision):
    n, T = 16, 24
    u0, ut = fields(n, 1), fields(n, 2)
    box = bgk.BGK3D(n, svisc=0.01, precision=precision)
    loss, g, gtau = adjoint(box, u0, ut, T, 5)
    rng = np.random.default_rng(3)
    du = rng.standard_normal((3, n, n, n))
    dtau = 0.7
    l2, dl = tangent(box, u0, du, dtau, ut, T)
    assert l2 == loss
    pred = float(np.dot(g, du.reshape(-1))) + gtau * dtau
    tol = 1e-9 if precision == "fp64" else 2e-4
    assert pred == pytest.approx(dl, rel=tol)
    box.close()


def test_adjoint_is_independent_of_checkpoint_interval(bgk):
    n, T = 12, 17
    u0, ut = fields(n, 4), fields(n, 5)
    box = bgk.BGK3D(n, svisc=0.02)
    ref = adjoint(box, u0, ut, T, T)
    for K in (1, 4, 6):
        got = adjoint(box, u0, ut, T, K)
        assert got[0] == ref[0] and got[2] == ref[2]
        assert np.array_equal(got[1], ref[1])
    box.close()


def test_adjoint_gradient_matches_central_differences_fp64(bgk):
    n, T, h = 16, 30, 1e-6
    u0, ut = fields(n, 6), fields(n, 7)
    box = bgk.BGK3D(n, svisc=0.01)
    loss, g, gtau = adjoint(box, u0, ut, T, 6)
    rng = np.random.default_rng(8)
    for _ in range(4):
        d = rng.standard_normal((3, n, n, n))
        d /= np.linalg.norm(d)
        lp = adjoint(box, u0 + h * d, ut, T, 6, grads=False)[0]
        lm = adjoint(box, u0 - h * d, ut, T, 6, grads=False)[0]
        fd = (lp - lm) / (2 * h)
        assert float(np.dot(g, d.reshape(-1))) == pytest.approx(fd, rel=1e-6)
    # tau: boxes with omega = 1/(tau +- h)
    om = box.omega
    tau = 1.0 / om
    ht = 1e-6
    lt = []
    for s in (1, -1):
        b2 = bgk.BGK3D(n, omega=1.0 / (tau + s * ht))
        lt.append(adjoint(b2, u0, ut, T, 6, grads=False)[0])
        b2.close()
    assert gtau == pytest.approx((lt[0] - lt[1]) / (2 * ht), rel=1e-5)
    box.close()


def test_adjoint_gradient_fp32_central_differences(bgk):
    n, T, h = 16, 20, 1e-3
    u0, ut = fields(n, 9), fields(n, 10)
    box = bgk.BGK3D(n, svisc=0.01, precision="fp32")
    _, g, _ = adjoint(box, u0, ut, T, 5)
    d = np.random.default_rng(11).standard_normal((3, n, n, n))
    d /= np.linalg.norm(d)
    lp = adjoint(box, u0 + h * d, ut, T, 5, grads=False)[0]
    lm = adjoint(box, u0 - h * d, ut, T, 5, grads=False)[0]
    assert float(np.dot(g, d.reshape(-1))) == pytest.approx((lp - lm) / (2 * h), rel=2e-3)
    box.close()


def _oracle_loss(O, u0, ut, T, svisc):
    n = u0[0].shape[0]
    L = O.OracleLattice(n, n, n)
    L.init_velocity(*u0, 1.0)
    for _ in range(T):
        L.step(svisc, periodic=True)
    d = L.get_dev()
    rho = d.sum(0) + 1.0
    cx = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], float)
    cy = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0], float)
    cz = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], float)
    u = [np.tensordot(c, d, 1) / rho for c in (cx, cy, cz)]
    return 0.5 * np.mean(sum((a - b) ** 2 for a, b in zip(u, ut)))


def test_adjoint_loss_and_gradient_against_cpu_oracle(bgk, oracle_mod):
    """Loss from the oracle's forward (bit-exact stepping) and central
    differences of it pin the GPU adjoint against an independent forward."""
    n, T, h = 8, 12, 1e-6
    u0, ut = fields(n, 12), fields(n, 13)
    box = bgk.BGK3D(n, svisc=0.01)
    loss, g, _ = adjoint(box, u0, ut, T, 4)
    assert loss == pytest.approx(_oracle_loss(oracle_mod, u0, ut, T, 0.01), rel=1e-12)
    d = np.random.default_rng(14).standard_normal((3, n, n, n))
    d /= np.linalg.norm(d)
    fd = (_oracle_loss(oracle_mod, [a + h * b for a, b in zip(u0, d)], ut, T, 0.01)
          - _oracle_loss(oracle_mod, [a - h * b for a, b in zip(u0, d)], ut, T, 0.01)) / (2 * h)
    assert float(np.dot(g, d.reshape(-1))) == pytest.approx(fd, rel=1e-6)
    box.close()


def test_adjoint_rejects_fp16_and_bad_arguments(bgk):
    n = 8
    u0 = fields(n, 1)
    box = bgk.BGK3D(n, precision="fp16")
    lib = box._lib
    loss = C.c_double()
    rc = lib.bgk_adjoint(box._h, _p(u0[0]), _p(u0[1]), _p(u0[2]), _p(u0[0]), _p(u0[1]), _p(u0[2]), 4, 2,
                         C.byref(loss), None, None)
    assert rc == bgk._abi.BGK_ERR_INVALID
    box.close()
    box = bgk.BGK3D(n)
    rc = box._lib.bgk_adjoint(box._h, _p(u0[0]), _p(u0[1]), _p(u0[2]), _p(u0[0]), _p(u0[1]), _p(u0[2]), 0, 2,
                              C.byref(loss), None, None)
    assert rc == bgk._abi.BGK_ERR_INVALID
    box.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_adjoint_state_cache_gives_identical_results(bgk, precision):
    """Keeping forward states (bgk_adjoint_cache) instead of recomputing them
    changes nothing in the loss or the gradients, whether some or all
    segments are kept; a budget of 0 frees the kept states."""
    n, T, K = 12, 17, 4
    u0, ut = fields(n, 4), fields(n, 5)
    box = bgk.BGK3D(n, svisc=0.02, precision=precision)
    ref = adjoint(box, u0, ut, T, K)
    es = 8 if precision == "fp64" else 4
    state = 19 * 32 * n * n * es  # rows padded to 32 cells
    lib = box._lib
    for budget in (state * (K - 1), 2 * state * (K - 1), 1 << 40):
        assert lib.bgk_adjoint_cache(box._h, budget) == 0
        got = adjoint(box, u0, ut, T, K)
        assert got[0] == ref[0] and got[2] == ref[2]
        assert np.array_equal(got[1], ref[1])
    before = box.device_bytes
    assert lib.bgk_adjoint_cache(box._h, 0) == 0
    assert box.device_bytes < before
    got = adjoint(box, u0, ut, T, K)
    assert np.array_equal(got[1], ref[1])
    box.close()


def test_adjoint_study_small_case(bgk):
    """The study driver behind the adjoint figures, at a small size: the
    gradient agrees with central differences (per-direction h-sweep) to 1e-6
    relative at the median and with the tangent-linear model to 1e-9."""
    from bgk3d_hit_b200 import adjoint_study

    r = adjoint_study.run(size=32, steps=60, ckpt=8, dirs=6, ntan=2, reps=1)
    assert r["fd_sweep"]["median_rel_err"] <= 1e-6, r["fd_sweep"]
    assert r["tangent"]["max_rel_err"] <= 1e-9, r["tangent"]
    assert r["fd"]["tau_rel_err"] <= 1e-5, r["fd"]
    assert r["loss"] == r["loss_in_adjoint_call"]


def _set_mode(box, mode):
    assert box._lib.bgk_adjoint_mode(box._h, mode) == 0, box._lib.bgk_last_error()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_adjoint_rebuild_matches_recompute(bgk, precision):
    """Rebuilding the forward states backwards (BGK_ADJ_REBUILD) gives the
    recomputed gradient up to the rounding of the rebuilt states: the loss is
    the same forward's, the gradients agree to 1e-11 (FP64) and 2e-5 (FP32)
    relative, in rel. L2 for dL/du0."""
    n, T, K = 16, 24, 6
    u0, ut = fields(n, 1), fields(n, 2)
    box = bgk.BGK3D(n, svisc=0.01, precision=precision)
    assert box._lib.bgk_adjoint_rebuilds(bgk._abi.PRECISIONS[precision], box.omega, K) == 1
    ref = adjoint(box, u0, ut, T, K)
    _set_mode(box, bgk._abi.BGK_ADJ_REBUILD)
    got = adjoint(box, u0, ut, T, K)
    tol = 1e-11 if precision == "fp64" else 2e-5
    assert got[0] == ref[0]
    assert _rel(got[1], ref[1]) <= tol
    assert got[2] == pytest.approx(ref[2], rel=tol)
    # T not a multiple of K, K = 1 (every step a first and last one), K = T
    for T2, K2 in ((23, 5), (7, 1), (9, 9)):
        _set_mode(box, bgk._abi.BGK_ADJ_RECOMPUTE)
        ref = adjoint(box, u0, ut, T2, K2)
        _set_mode(box, bgk._abi.BGK_ADJ_REBUILD)
        got = adjoint(box, u0, ut, T2, K2)
        assert got[0] == ref[0]
        assert _rel(got[1], ref[1]) <= tol, (T2, K2)
        assert got[2] == pytest.approx(ref[2], rel=tol)
    box.close()


def test_adjoint_rebuild_matches_tangent_linear(bgk):
    """Dot-product test of the rebuilt-state adjoint against the tangent
    model along the stored forward trajectory, 1e-9 relative (FP64)."""
    n, T = 16, 24
    u0, ut = fields(n, 1), fields(n, 2)
    box = bgk.BGK3D(n, svisc=0.01)
    _set_mode(box, bgk._abi.BGK_ADJ_REBUILD)
    loss, g, gtau = adjoint(box, u0, ut, T, 8)
    du = np.random.default_rng(3).standard_normal((3, n, n, n))
    dtau = 0.7
    _, dl = tangent(box, u0, du, dtau, ut, T)
    assert float(np.dot(g, du.reshape(-1))) + gtau * dtau == pytest.approx(dl, rel=1e-9)
    box.close()


def test_adjoint_rebuild_with_state_cache_and_rule(bgk):
    """Cached segments use their kept states and the others are rebuilt; where
    |1 - omega|^-(K-1) > 64 (omega = 1.25, K = 6) the call recomputes, and
    then its results equal the recompute mode's bit for bit."""
    n, T, K = 12, 17, 4
    u0, ut = fields(n, 4), fields(n, 5)
    box = bgk.BGK3D(n, svisc=0.02)
    lib = box._lib
    ref = adjoint(box, u0, ut, T, K)
    _set_mode(box, bgk._abi.BGK_ADJ_REBUILD)
    state = 19 * 32 * n * n * 8
    assert lib.bgk_adjoint_cache(box._h, 2 * state * (K - 1)) == 0
    got = adjoint(box, u0, ut, T, K)
    assert got[0] == ref[0] and _rel(got[1], ref[1]) <= 1e-11
    assert lib.bgk_adjoint_cache(box._h, 0) == 0
    box.close()
    box = bgk.BGK3D(n, omega=1.25)
    lib = box._lib
    assert lib.bgk_adjoint_rebuilds(0, 1.25, 6) == 0 and lib.bgk_adjoint_rebuilds(0, 1.25, 3) == 1
    ref = adjoint(box, u0, ut, T, 6)
    _set_mode(box, bgk._abi.BGK_ADJ_REBUILD)
    got = adjoint(box, u0, ut, T, 6)
    assert got[0] == ref[0] and got[2] == ref[2] and np.array_equal(got[1], ref[1])
    assert lib.bgk_adjoint_mode(box._h, 7) == bgk._abi.BGK_ERR_INVALID
    box.close()
