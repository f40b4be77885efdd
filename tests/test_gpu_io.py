"""GPU tests of the file outputs: checkpoint / restart (bgk_save, bgk_load)
and the VTK writer (bgk_vtk) against the reference's vtk_*_bin layout."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], float)
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0], float)
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], float)


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("schemes", [("two_lattice", "two_lattice"), ("aa", "two_lattice"), ("two_lattice", "aa"),
                                     ("aa", "aa")])
def test_restart_continues_bit_exact(bgk, tmp_path, form, schemes):
    shape = (24, 20, 16)
    a = bgk.BGK3D(*shape, precision=form, scheme=schemes[0], svisc=0.01, u0=0.05)
    a.init()
    a.run(7)
    path = str(tmp_path / "restart.bin")
    a.save(path)
    a.run(5)
    ref = a.populations()
    b = bgk.BGK3D(*shape, precision=form, scheme=schemes[1], svisc=0.01, u0=0.05)
    b.load(path)
    assert b.step == 7 and b.scale == a.scale
    b.run(5)
    assert b.step == 12
    assert same_bits(b.populations(), ref)
    a.close()
    b.close()


def test_restart_rejects_mismatched_or_bad_files(bgk, tmp_path):
    a = bgk.BGK3D(16, precision="fp64")
    a.init()
    p = str(tmp_path / "r.bin")
    a.save(p)
    for kw in (dict(lx=18), dict(precision="fp32")):
        args = dict(lx=16, precision="fp64")
        args.update(kw)
        b = bgk.BGK3D(args["lx"], 16, 16, precision=args["precision"])
        with pytest.raises(bgk.BgkError) as e:
            b.load(p)
        assert e.value.code == bgk._abi.BGK_ERR_INVALID
        b.close()
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not a checkpoint" * 4)
    with pytest.raises(bgk.BgkError):
        a.load(str(bad))
    trunc = tmp_path / "trunc.bin"
    trunc.write_bytes(open(p, "rb").read()[:1000])
    with pytest.raises(bgk.BgkError):
        a.load(str(trunc))
    a.close()


def _read_vtk(path):
    raw = open(path, "rb").read()
    lines, pos = [], 0
    for _ in range(9):
        end = raw.index(b"\n", pos)
        lines.append(raw[pos:end].decode())
        pos = end + 1
    data = np.frombuffer(raw[pos:], dtype=">f4").astype(np.float32)
    return lines, data


def _velocity_f32(dev):
    """u = j/rho as the reference's VTK writers form it: sums in the storage
    arithmetic (double here), rounded to single precision, divided in single."""
    den = (dev.sum(0) + 1.0).astype(np.float32)
    return [(np.tensordot(c, dev, 1)).astype(np.float32) / den for c in (CX, CY, CZ)]


@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
def test_vtk_slices_and_box_match_reference_layout(bgk, tmp_path, scheme):
    nx, ny, nz = 12, 10, 8
    box = bgk.BGK3D(nx, ny, nz, svisc=0.01, u0=0.05, scheme=scheme)
    box.init()
    box.run(3)
    u = _velocity_f32(box.deviations())  # each (nz, ny, nx)
    d = str(tmp_path)
    box.vtk_xy_bin(3, 4, d)
    box.vtk_xz_bin(3, 5, d)
    box.vtk_yz_bin(3, 6, d)
    box.vtk_3d_bin(3, d)
    cases = {
        "xy": ((nx, ny, 1), (1, 1, 4), [c[3] for c in u]),
        "xz": ((nx, 1, nz), (1, 5, 1), [c[:, 4, :] for c in u]),
        "yz": ((1, ny, nz), (6, 1, 1), [c[:, :, 5] for c in u]),
        "3d": ((nx, ny, nz), (1, 1, 1), u),
    }
    for tag, (dims, orig, comp) in cases.items():
        lines, data = _read_vtk(f"{d}/tec_{tag}.00000.00000003.vtk")
        npts = dims[0] * dims[1] * dims[2]
        assert lines == ["# vtk DataFile Version 2.0", "Campo", "BINARY", "DATASET STRUCTURED_POINTS",
                         "DIMENSIONS %10d %10d %10d" % dims, "ORIGIN %10d %10d %10d" % orig,
                         "SPACING %10d %10d %10d" % (1, 1, 1), "POINT_DATA%10d" % npts, "VECTORS velocity float "]
        exp = np.stack([c.reshape(-1) for c in comp], axis=1).reshape(-1)
        assert data.size == 3 * npts
        np.testing.assert_allclose(data, exp, rtol=2.5e-7, atol=1e-12)
    with pytest.raises(bgk.BgkError):
        box.vtk_xy_bin(3, nz + 1, d)
    box.close()


def test_run_loop_writes_slices_and_restarts(bgk, tmp_path):
    from bgk3d_hit_b200 import run_loop

    box = bgk.BGK3D(16, svisc=0.01, u0=0.05, icheck=5)
    box.init()
    run_loop(box, 10, str(tmp_path), ivtim=10, itsave=5)
    names = sorted(p.name for p in tmp_path.iterdir())
    for it in (0, 10):
        for tag in ("xy", "xz", "yz"):
            assert f"tec_{tag}.00000.{it:08d}.vtk" in names
    assert "restart.00000005.bin" in names and "restart.00000010.bin" in names
    box.close()


def test_program_driver_matches_run_loop(bgk, tmp_path):
    """The C++ driver bgk3d_hit (namelist in, diagno.dat / dissipation.dat /
    VTK / restarts out) writes the same files as run_loop for the same run."""
    import subprocess

    from bgk3d_hit_b200 import build as B
    from bgk3d_hit_b200 import run_loop

    exe = B.build_driver()
    (tmp_path / "c").mkdir()
    (tmp_path / "py").mkdir()
    nl = tmp_path / "bgk.input"
    nl.write_text("&parameters\nlx = 16\nly = 12\nlz = 10\nu0 = 0.05\nsvisc = 0.01\n"
                  "itfin = 20\nitsave = 10\nivtim = 10\nicheck = 5 /\n")
    r = subprocess.run([exe, str(nl), "--out", str(tmp_path / "c")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "GLUPS" in r.stdout
    box = bgk.BGK3D.from_input(str(nl), mode="faithful")
    box.init()
    run_loop(box, 20, str(tmp_path / "py"), ivtim=10, itsave=10)
    box.close()
    for name in ("diagno.dat", "dissipation.dat", "tec_xy.00000.00000010.vtk", "restart.00000020.bin"):
        assert (tmp_path / "c" / name).read_bytes() == (tmp_path / "py" / name).read_bytes(), name
    assert (tmp_path / "c" / "bgk.perf").exists()
