"""GPU tests of the z-slab decomposition (proc_z > 1): slabs that exchange
their face populations through each other's ghost planes must reproduce the
whole periodic box bit for bit, in every form, with and without the LES
collision; their diagnostics must sum to the whole box's (compensated FP64
sums in a different order: 1e-12 relative).

All slabs run on the one GPU of the test: in one process (LocalSlabs, the
ghost buffers shared as plain device pointers) and in two processes (CUDA IPC
handles, a host barrier between steps). No kernel waits on another; the
barrier is on the host."""
import os

import numpy as np
import pytest

from test_gpu_parity import F16_SCALE, same_bits

pytestmark = pytest.mark.gpu


def _kw(form, **kw):
    d = dict(svisc=0.01, u0=0.05, precision=form, icheck=1)
    if form == "fp16":
        d["fp16_scale"] = F16_SCALE
    d.update(kw)
    return d


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("proc_z", [2, 3, 4])
@pytest.mark.parametrize("les_cs", [0.0, 0.17])
@pytest.mark.parametrize("nx", [20, 32])  # 32: FP16 / FP32 interior planes on the four- / two-cells-per-thread kernels
def test_local_slabs_bitexact_vs_whole_box(bgk, form, proc_z, les_cs, nx):
    from bgk3d_hit_b200.slabs import LocalSlabs

    shape = (nx, 12, 24)
    box = bgk.BGK3D(*shape, **_kw(form, les_cs=les_cs))
    box.init()
    sl = LocalSlabs(*shape, proc_z, **_kw(form, les_cs=les_cs))
    sl.init()
    assert same_bits(sl.populations(), box.populations()), "TGV init with global z"
    for it in range(1, 7):
        box.col_MC(it)
        sl.step(it)
        if it in (1, 6):
            assert same_bits(sl.populations(), box.populations()), f"after {it} steps"
    sl.close()
    box.close()


def test_local_slabs_velocity_init_and_one_plane_slabs(bgk):
    from bgk3d_hit_b200.hit import hit_velocity
    from bgk3d_hit_b200.slabs import LocalSlabs

    n = 16
    u = hit_velocity(n, 2, 0.05, 3)
    for proc_z in (4, 16):  # 16: one plane per slab, both faces on the same plane
        sl = LocalSlabs(n, n, n, proc_z, **_kw("fp64"))
        sl.init_velocity(*u)
        b = bgk.BGK3D(n, **_kw("fp64"))
        b.init_velocity(*u)
        for it in range(1, 5):
            sl.step(it)
            b.col_MC(it)
        assert same_bits(sl.populations(), b.populations()), proc_z
        sl.close()
        b.close()


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
def test_slab_diagnostics_sum_to_whole_box(bgk, form):
    from bgk3d_hit_b200.slabs import LocalSlabs

    shape = (16, 16, 24)
    box = bgk.BGK3D(*shape, **_kw(form))
    box.init()
    sl = LocalSlabs(*shape, 3, **_kw(form))
    sl.init()
    for it in range(1, 4):
        box.col_MC(it)
        sl.step(it)
    ref = box.diagnostic(3)
    got = sl.diagnostic(3)
    for k in ("rho_mean", "ke_mean", "tke_norm", "diss", "tke", "eps_strain"):
        assert got[k] == pytest.approx(ref[k], rel=1e-12), k
    for k in ("ux_mean", "uy_mean", "uz_mean"):
        assert got[k] == pytest.approx(ref[k], rel=1e-10, abs=1e-18), k
    assert got["t"] == ref["t"] and got["nonfinite"] == 0
    sl.close()
    box.close()


def test_slab_restart_and_vtk(bgk, tmp_path):
    from bgk3d_hit_b200.slabs import LocalSlabs

    shape = (12, 10, 8)
    sl = LocalSlabs(*shape, 2, **_kw("fp64"))
    sl.init()
    sl.run(3)
    for r, s in enumerate(sl.slabs):
        s.save(str(tmp_path / f"restart.{r}.bin"))
    sl.run(4)
    ref = sl.populations()
    sl2 = LocalSlabs(*shape, 2, **_kw("fp64"))
    for r, s in enumerate(sl2.slabs):
        s.load(str(tmp_path / f"restart.{r}.bin"))
    sl2.prime()
    sl2.run(4)
    assert same_bits(sl2.populations(), ref)
    # per-rank VTK files with the slab's z offset (SRC/vtk_xy.binary.F90:53,65-67)
    sl2.slabs[1].vtk_xy_bin(7, 2, str(tmp_path))
    sl2.slabs[1].vtk_3d_bin(7, str(tmp_path))
    head = open(tmp_path / "tec_xy.00001.00000007.vtk", "rb").read().split(b"\n")[:6]
    assert head[4] == b"DIMENSIONS %10d %10d %10d" % (12, 10, 1)
    assert head[5] == b"ORIGIN %10d %10d %10d" % (1, 1, 4 + 2)
    head = open(tmp_path / "tec_3d.00001.00000007.vtk", "rb").read().split(b"\n")[:6]
    assert head[4] == b"DIMENSIONS %10d %10d %10d" % (12, 10, 4)
    assert head[5] == b"ORIGIN %10d %10d %10d" % (1, 1, 5)
    sl.close()
    sl2.close()


def test_slab_call_order_and_unsupported_calls(bgk):
    import ctypes as C

    lib = bgk.load()
    s = bgk.BGK3D(8, 8, 8, proc_z=2, coord_z=0, **_kw("fp64"))
    s.init()
    assert lib.bgk_col_mc(s._h, 1) == bgk._abi.BGK_ERR_STATE  # not connected
    buf, nbytes = s.halo_buffer()
    assert nbytes == 2 * 2 * 5 * 256 * 8  # 2 parities x 2 faces x 5 pops x padded 8x8 plane, FP64
    s.halo_connect(buf, buf)
    assert lib.bgk_col_mc(s._h, 1) == bgk._abi.BGK_ERR_STATE  # not primed
    s.halo_prime()
    assert lib.bgk_run(s._h, 2) == bgk._abi.BGK_ERR_INVALID
    assert lib.bgk_spectrum(s._h, 4, (C.c_double * 4)()) == bgk._abi.BGK_ERR_INVALID
    s.init()  # a new state needs a new prime
    assert lib.bgk_col_mc(s._h, 1) == bgk._abi.BGK_ERR_STATE
    s.close()
    w = bgk.BGK3D(8)
    with pytest.raises(bgk.BgkError):
        w.halo_buffer()
    w.close()


def test_slab_edge_kernel_time(bgk):
    """The edge-plane kernel of a slab step is timed on the device: an error
    before the first step, a positive duration shorter than the whole step
    after it, and an error on a whole-box context."""
    from bgk3d_hit_b200.slabs import LocalSlabs

    sl = LocalSlabs(64, 64, 64, 2, svisc=0.01, u0=0.05, icheck=1)
    try:
        sl.init()
        with pytest.raises(bgk.BgkError):
            sl.slabs[0].slab_edge_time_us()
        sl.run(3)
        for s in sl.slabs:
            us = s.slab_edge_time_us()
            assert 0.0 < us < 1e5
    finally:
        sl.close()
    w = bgk.BGK3D(8)
    with pytest.raises(bgk.BgkError):
        w.slab_edge_time_us()
    w.close()


def _two_process_worker(rank, port, out_dir, steps):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        from bgk3d_hit_b200.slabs import DistSlabs

        ds = DistSlabs(16, 12, 20, device=0, svisc=0.01, u0=0.05, icheck=1)
        ds.init()
        for it in range(1, steps + 1):
            ds.step(it)
        d = ds.diagnostic(steps)
        np.save(os.path.join(out_dir, f"slab{rank}.npy"), ds.box.populations())
        np.save(os.path.join(out_dir, f"diag{rank}.npy"), np.array([d["ke_mean"], d["diss"]]))
        ds.close()
    finally:
        dist.destroy_process_group()


def test_two_processes_share_ghost_planes_by_ipc(bgk, tmp_path):
    """Two slab processes on this GPU, ghost buffers exchanged as CUDA IPC
    handles, gloo host barrier: bit-exact with the whole box."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    steps = 5
    mp.start_processes(_two_process_worker, args=(port, str(tmp_path), steps), nprocs=2, join=True,
                       start_method="spawn")
    got = np.concatenate([np.load(tmp_path / f"slab{r}.npy") for r in range(2)], axis=1)
    box = bgk.BGK3D(16, 12, 20, svisc=0.01, u0=0.05, icheck=1)
    box.init()
    box.run(steps)
    assert same_bits(got, box.populations())
    ref = box.diagnostic(steps)
    for r in range(2):
        ke, diss = np.load(tmp_path / f"diag{r}.npy")
        assert ke == pytest.approx(ref["ke_mean"], rel=1e-12)
        assert diss == pytest.approx(ref["diss"], rel=1e-12)
    box.close()
