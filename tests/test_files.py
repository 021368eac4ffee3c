"""The reference's files through the C ABI (host code; no device needed):
.turbb parameters as initparams reads them (params.f90:119-207 through
miscel.f90:13-262), snapshots in the layout of output_data / read_input_data
(input_output.f90:288-680) and the Lund means file."""
import os
import struct

import numpy as np
import pytest

from blgpu import files, BlgpuError

# the reference source tree (its .turbb files), when present on this machine
REF = os.environ.get("BLGPU_REFERENCE_DIR", "")


def write_turbb(path, text):
    path.write_text(text)
    return str(path)


def test_turbb_syntax(tmp_path):
    f = write_turbb(tmp_path / "a.turbb", "\n".join([
        "! comment line, nu = 7 is not read",
        "nxyz = 34 17 12 ! (*) trailing comment",
        "!WM = 3",
        "  nu   =  1.5d-5",
        "CFL = -2E-3",
        "nu = 9.0             ! a second nu: the first line wins",
        "RKscheme = 3",
        "boxsize = 10.0, 0.5 ,0.2 3.",
        "alphas = 5*0.25",
        "inflow_file =./profiles/blasius.dat",
        "fileout = out/BL ! where to write",
        "init_rand = 1",
        "LES =",                      # blank value: absent
        "WMnut = 0.05",
        "line without an equals sign",
    ]))
    p = files.read_params(f)
    assert p["nxyz"] == [34, 17, 12]
    assert p["nu"] == 1.5e-5 and p["CFL"] == -2e-3 and p["RKscheme"] == 3
    assert p["boxsize"] == [10.0, 0.5, 0.2, 3.0]
    assert p["alphas"] == [0.25] * 5
    assert p["inflow_file"] == "./profiles/blasius.dat" and p["fileout"] == "out/BL"
    assert "WM" not in p and "LES" not in p and "filein" not in p
    assert p["WMnut"] == 0.05
    assert p["init_step"] == -45  # not given
    assert p["config"] == dict(nx=34, ny=17, nz=12, nu=1.5e-5, cfl=-2e-3, dpdx=0.0, dpdz=0.0, rk_scheme=3,
                               les_model=0)


def test_turbb_errors(tmp_path):
    with pytest.raises(BlgpuError, match="does not exist"):
        files.read_params(tmp_path / "missing.turbb")
    with pytest.raises(BlgpuError, match="inflow_file"):
        files.read_params(write_turbb(tmp_path / "b.turbb", "nxyz = 4 4 4\n"))
    with pytest.raises(BlgpuError, match="init_rand = 1, but filein exists"):
        files.read_params(write_turbb(tmp_path / "c.turbb", "inflow_file = a\ninit_rand = 1\nfilein = x\n"))
    with pytest.raises(BlgpuError, match="not an integer"):
        files.read_params(write_turbb(tmp_path / "d.turbb", "inflow_file = a\nnsteps = 1e3\n"))
    with pytest.raises(BlgpuError, match="expected 3"):
        files.read_params(write_turbb(tmp_path / "e.turbb", "inflow_file = a\nnxyz = 4 4\n"))


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="BLGPU_REFERENCE_DIR not set")
def test_reference_turbb_files():
    p = files.read_params(os.path.join(REF, "laminar_test", "laminar.turbb"))
    assert p["nxyz"] == [302, 64, 8] and p["CFL"] == -5e-5 and p["nu"] == 1e-5
    assert p["RKscheme"] == 2 and p["init_rand"] == 1 and p["inflow_flag"] == 1 and p["top_flag"] == 0
    assert p["boxsize"] == [10.0, 0.10, 0.2, 3.0]
    assert p["inflow_file"] == "blasius_solution.dat" and p["fileout"] == "./data/BL_laminar"
    q = files.read_params(os.path.join(REF, "tests", "test.turbb"))
    assert q["nxyz"] == [1156, 192, 34] and q["inflow_flag"] == 5 and q["LES"] == 1
    assert q["Lund_ix"] == 200 and q["Lund_deltai"] == 0.024998 and q["Lund_T"] == 0.5
    assert q["filein"] == "./data/test_swap.00500000" and q["init_step"] == 500000
    r = files.read_params(os.path.join(REF, "transition_test", "transition.turbb"))
    assert r["nxyz"] == [814, 125, 66] and r["Amplitude"] == 0.20
    assert r["timeinflow_file"] == "temporal_modes_inlet.dat"


def box(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    nxg, nyg, nzg = nx + 1, ny + 1, nz + 1
    x = 1.0 + np.cumsum(rng.uniform(0.5, 1.5, nx)) - 0.75
    y = np.concatenate([[0.0], np.cumsum(rng.uniform(0.1, 1.0, ny - 1))])
    z = np.linspace(0.0, 3.0, nz)
    U = np.asfortranarray(rng.standard_normal((nx, nyg, nzg)))
    V = np.asfortranarray(rng.standard_normal((nxg, ny, nzg)))
    W = np.asfortranarray(rng.standard_normal((nxg, nyg, nz)))
    nt = np.asfortranarray(rng.standard_normal((nxg, nyg, nzg)))
    P = np.asfortranarray(rng.standard_normal((nxg, nyg, nzg)))
    return x, y, z, U, V, W, nt, P


def reader_one_process(path):
    """The snapshot layout restated in numpy: the reference's GPU runs write
    n3-1 z-planes of U, V, W (and nu_t) after their 3 dims, P in full."""
    with open(path, "rb") as f:
        t, nu = struct.unpack("dd", f.read(16))
        magic, step = struct.unpack("ii", f.read(8))
        mesh = []
        for _ in range(6):
            n = struct.unpack("i", f.read(4))[0]
            mesh.append(np.frombuffer(f.read(8 * n), dtype="<f8"))
        fields = []
        for q in range(5):
            n1, n2, n3 = struct.unpack("iii", f.read(12))
            n3a = n3 if q == 4 else n3 - 1
            a = np.frombuffer(f.read(8 * n1 * n2 * n3a), dtype="<f8").reshape((n3a, n2, n1)).transpose(2, 1, 0)
            fields.append(a)
        assert f.read() == b""
    return t, nu, magic, step, mesh, fields


def test_snapshot_layout_and_round_trip(tmp_path):
    nx, ny, nz = 9, 7, 6
    x, y, z, U, V, W, nt, P = box(nx, ny, nz, 1)
    path = tmp_path / "BL.00000042"
    files.write_snapshot(path, 1.25, 1e-5, 42, x, y, z, U, V, W, nt, P)
    t, nu, magic, step, mesh, fl = reader_one_process(path)
    assert (t, nu, magic, step) == (1.25, 1e-5, -73, 42)
    assert np.array_equal(mesh[0], x) and np.array_equal(mesh[1], y) and np.array_equal(mesh[2], z)
    for m, f in zip(mesh[3:], (x, y, z)):
        assert np.array_equal(m, 0.5 * (f[:-1] + f[1:]))  # initialization.f90:181-189
    assert np.array_equal(fl[0], U[:, :, :-1]) and np.array_equal(fl[1], V[:, :, :-1])
    assert np.array_equal(fl[2], W[:, :, :-1]) and np.array_equal(fl[3], nt[:, :, :-1])
    assert np.array_equal(fl[4], P)
    s = files.read_snapshot(path)
    assert s["step"] == 42 and s["t"] == 1.25 and s["full_planes"] == 0 and s["has_nu_t_p"] == 1
    assert np.array_equal(s["x"], x) and np.array_equal(s["y"], y) and np.array_equal(s["z"], z)
    # the plane left out comes back as the z-periodic boundary pass sets it
    for got, ref, face in ((s["U"], U, False), (s["V"], V, False), (s["W"], W, True), (s["nu_t"], nt, False)):
        assert np.array_equal(got[:, :, :-1], ref[:, :, :-1])
        assert np.array_equal(got[:, :, -1], ref[:, :, 1 if face else 2])
    assert np.array_equal(s["P"], P)


def write_full(path, t, nu, step, x, y, z, fields, magic=True, tail=True, order="<"):
    with open(path, "wb") as f:
        f.write(struct.pack(order + "dd", t, nu))
        if magic:
            f.write(struct.pack(order + "ii", -73, step))
        for a in (x, y, z, 0.5 * (x[:-1] + x[1:]), 0.5 * (y[:-1] + y[1:]), 0.5 * (z[:-1] + z[1:])):
            f.write(struct.pack(order + "i", len(a)) + np.asarray(a, order + "f8").tobytes())
        for a in (fields if tail else fields[:3]):
            f.write(struct.pack(order + "iii", *a.shape) + np.asarray(a, order + "f8").tobytes(order="F"))


def test_snapshot_full_layout_and_older_files(tmp_path):
    nx, ny, nz = 8, 6, 7
    x, y, z, U, V, W, nt, P = box(nx, ny, nz, 2)
    path = tmp_path / "full"
    write_full(path, 0.5, 2e-5, 7, x, y, z, [U, V, W, nt, P])
    s = files.read_snapshot(path)
    assert s["full_planes"] == 1 and s["step"] == 7
    for k, a in zip(("U", "V", "W", "nu_t", "P"), (U, V, W, nt, P)):
        assert np.array_equal(s[k], a)
    # no magic number (older files) and no nu_t / P records
    path2 = tmp_path / "old"
    write_full(path2, 0.5, 2e-5, 0, x, y, z, [U, V, W, nt, P], magic=False, tail=False)
    s2 = files.read_snapshot(path2)
    assert s2["step"] == -1 and s2["has_nu_t_p"] == 0
    assert np.array_equal(s2["U"], U) and not s2["P"].any() and not s2["nu_t"].any()


def test_snapshot_errors(tmp_path):
    nx, ny, nz = 8, 6, 7
    x, y, z, U, V, W, nt, P = box(nx, ny, nz, 3)
    path = tmp_path / "s"
    files.write_snapshot(path, 0.0, 1e-5, 0, x, y, z, U, V, W, nt, P)
    data = path.read_bytes()
    (tmp_path / "cut").write_bytes(data[:-8])
    with pytest.raises(BlgpuError, match="fit neither"):
        files.read_snapshot(tmp_path / "cut")
    with pytest.raises(BlgpuError, match="cannot open"):
        files.read_snapshot(tmp_path / "none")


def test_rescaling_means_either_byte_order(tmp_path):
    rng = np.random.default_rng(4)
    ny = 9
    um, vm = rng.standard_normal(ny + 1), rng.standard_normal(ny)
    files.write_rescaling(tmp_path / "m", um, vm)
    raw = (tmp_path / "m").read_bytes()
    assert raw == struct.pack("<i", ny + 1) + um.astype("<f8").tobytes() + vm.astype("<f8").tobytes()
    a, b = files.read_rescaling(tmp_path / "m", ny)
    assert np.array_equal(a, um) and np.array_equal(b, vm)
    # big-endian, as read_input_data opens it (input_output.f90:445)
    (tmp_path / "be").write_bytes(struct.pack(">i", ny + 1) + um.astype(">f8").tobytes() + vm.astype(">f8").tobytes())
    a, b = files.read_rescaling(tmp_path / "be", ny)
    assert np.array_equal(a, um) and np.array_equal(b, vm)
    with pytest.raises(BlgpuError, match="nyg_resc"):
        files.read_rescaling(tmp_path / "m", ny + 1)


def test_snapshot_name():
    assert files.snapshot_name("./data/BL", 500) == "./data/BL.00000500"
    assert files.snapshot_name("  out/x ", 123456789) == "out/x.123456789"


def test_params_les_flag_maps_to_config(tmp_path):
    """The .turbb LES flag goes to blgpu_config.les_model unchanged (2: the
    dynamic model with the coefficient averaged in z)."""
    p = files.read_params(write_turbb(tmp_path / "l.turbb", "inflow_file = a\nLES = 2\n"))
    assert p["LES"] == 2 and p["config"]["les_model"] == 2


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "inflow_profiles_ref.json")


def _write_profile(path, ny, U, V, order):
    with open(path, "wb") as f:
        f.write(struct.pack(order + "i", ny))
        f.write(np.asarray(U, dtype=order + "f8").tobytes())
        f.write(np.asarray(V, dtype=order + "f8").tobytes())
    return str(path)


def test_inflow_profiles_of_the_reference(tmp_path):
    """inflow_file of inflow flags 2 and 5 (boundary_conditions.f90:1405-1413,
    1550-1558): the reference's two profile files, one little- and one
    big-endian (tests/golden/inflow_profiles_ref.json, decoded from them by
    make_golden.py), written back in their byte order and read through the C
    ABI to the bit; the file's ny must equal the grid's."""
    import json
    profs = json.load(open(GOLDEN))
    assert {p["order"] for p in profs} == {"little", "big"}
    for p in profs:
        ny = p["ny"]
        f = _write_profile(tmp_path / os.path.basename(p["source"]), ny, p["U_inlet"], p["V_inlet"],
                           "<" if p["order"] == "little" else ">")
        assert os.path.getsize(f) == p["bytes"]
        U, V = files.read_inflow_profile(f)
        assert U.shape == (ny + 1,) and V.shape == (ny,)
        assert np.array_equal(U, np.array(p["U_inlet"])) and np.array_equal(V, np.array(p["V_inlet"]))
        U2, V2 = files.read_inflow_profile(f, ny)
        assert np.array_equal(U, U2) and np.array_equal(V, V2)
        with pytest.raises(BlgpuError, match="Profile doesnt match dimensions"):
            files.read_inflow_profile(f, ny + 1)


def test_inflow_profile_errors(tmp_path):
    f = _write_profile(tmp_path / "short.dat", 8, np.ones(9), np.ones(7), "<")  # one V value missing
    with pytest.raises(BlgpuError, match="not an inflow profile"):
        files.read_inflow_profile(f)
    with pytest.raises(BlgpuError, match="cannot open"):
        files.read_inflow_profile(str(tmp_path / "absent.dat"))


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="BLGPU_REFERENCE_DIR not set")
def test_inflow_profile_files_in_the_reference_tree():
    """The profiles read straight from the reference tree equal the golden
    fixture (which pins the fixture to the files)."""
    import hashlib
    import json
    for p in json.load(open(GOLDEN)):
        path = os.path.join(REF, p["source"])
        assert hashlib.sha256(open(path, "rb").read()).hexdigest() == p["sha256"]
        U, V = files.read_inflow_profile(path)
        assert np.array_equal(U, np.array(p["U_inlet"])) and np.array_equal(V, np.array(p["V_inlet"]))


def test_snapshot_big_endian_files(tmp_path):
    """The reference's GPU build runs with F_UFMTENDIAN=big (its Makefile
    exports it), so its snapshots are big-endian: read in either order, the
    order told by which one gives a consistent header and layout (sizes
    such as nx = 512 look plausible in both orders; the layout decides)."""
    for nx, ny, nz in ((8, 6, 7), (512, 3, 3)):
        x, y, z, U, V, W, nt, P = box(nx, ny, nz, 5)
        for magic, tail in ((True, True), (False, False)):
            path = tmp_path / ("be_%d_%d" % (nx, magic))
            write_full(path, 0.75, 3e-5, 11, x, y, z, [U, V, W, nt, P], magic=magic, tail=tail, order=">")
            s = files.read_snapshot(path)
            assert s["t"] == 0.75 and s["step"] == (11 if magic else -1) and s["full_planes"] == 1
            assert np.array_equal(s["x"], x) and np.array_equal(s["z"], z)
            for k, a in (zip(("U", "V", "W", "nu_t", "P"), (U, V, W, nt, P)) if tail else
                         zip(("U", "V", "W"), (U, V, W))):
                assert np.array_equal(s[k], a)


def test_writers_follow_F_UFMTENDIAN(tmp_path, monkeypatch):
    """F_UFMTENDIAN=big makes the snapshot and Lund-means writers big-endian,
    as the NVHPC runtime does for the reference's files; the readers take
    the result back to the bit; a unit list leaves the native order."""
    nx, ny, nz = 9, 7, 6
    x, y, z, U, V, W, nt, P = box(nx, ny, nz, 6)
    files.write_snapshot(tmp_path / "le", 1.5, 1e-5, 3, x, y, z, U, V, W, nt, P)
    monkeypatch.setenv("F_UFMTENDIAN", "big")
    files.write_snapshot(tmp_path / "be", 1.5, 1e-5, 3, x, y, z, U, V, W, nt, P)
    um, vm = np.linspace(0.0, 1.0, ny + 1), np.linspace(-1.0, 0.0, ny)
    files.write_rescaling(tmp_path / "mbe", um, vm)
    monkeypatch.setenv("F_UFMTENDIAN", "big:10,11")
    files.write_rescaling(tmp_path / "mle", um, vm)
    monkeypatch.delenv("F_UFMTENDIAN")
    le, be = (tmp_path / "le").read_bytes(), (tmp_path / "be").read_bytes()
    assert len(le) == len(be) and le != be
    assert struct.unpack(">2d2i", be[:24]) == (1.5, 1e-5, -73, 3)
    a, b = files.read_snapshot(tmp_path / "le"), files.read_snapshot(tmp_path / "be")
    for k in ("x", "y", "z", "U", "V", "W", "nu_t", "P"):
        assert np.array_equal(a[k], b[k])
    assert (tmp_path / "mbe").read_bytes() == struct.pack(">i", ny + 1) + um.astype(">f8").tobytes() + \
        vm.astype(">f8").tobytes()
    assert (tmp_path / "mle").read_bytes() == struct.pack("<i", ny + 1) + um.astype("<f8").tobytes() + \
        vm.astype("<f8").tobytes()
    for f in ("mbe", "mle"):
        c, d = files.read_rescaling(tmp_path / f, ny)
        assert np.array_equal(c, um) and np.array_equal(d, vm)


def test_statistics_text_layout(tmp_path):
    """output_statistics (input_output.f90:685-746): '%' and t, nu in F15.8,
    nx, ny, nz, istep in I8; Cf, x, y one record each; then the eight means
    as nx records of ny F15.8 values (UVmean is not written)."""
    rng = np.random.default_rng(8)
    nx, ny = 5, 4
    x, y = np.linspace(0.0, 2.0, nx), np.linspace(0.0, 1.0, ny)
    Cf = rng.uniform(-1e-3, 5e-3, nx)
    Cf[1], Cf[2], Cf[3] = 1.0e7, np.nan, -0.0
    means = rng.standard_normal((9, nx, ny))
    p = tmp_path / "s.stats.txt"
    files.write_statistics(p, 1.5, 1e-5, 6, 7, Cf, x, y, means)
    lines = p.read_text().splitlines()
    assert lines[0] == "%     1.50000000     0.00001000       5       4       6       7"
    assert len(lines) == 4 + 8 * nx
    assert lines[1][15:30] == "*" * 15 and lines[1][30:45] == " " * 12 + "NaN"
    assert lines[1][45:60] == "    -0.00000000"
    assert all(len(l) == 15 * nx for l in lines[1:3]) and len(lines[3]) == 15 * ny
    assert all(len(l) == 15 * ny for l in lines[4:])
    s = files.read_statistics(p)
    assert (s["t"], s["nu"], s["nx"], s["ny"], s["nz"], s["istep"]) == (1.5, 1e-5, 5, 4, 6, 7)
    assert np.array_equal(s["x"], np.round(x, 8)) and np.array_equal(s["y"], np.round(y, 8))
    for q, name in zip((0, 1, 2, 3, 4, 5, 7, 8),
                       ("Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "Pmean", "P2mean")):
        assert np.abs(s[name] - means[q]).max() <= 5.01e-9, name
