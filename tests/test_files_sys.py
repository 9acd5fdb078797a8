"""The reference's binary formats (lib/files_sys) read and written by
radrhd_solver_b200.files_sys.  CPU only.

The golden files under tests/golden/files_sys/ were written by the reference's
own WriteGridGeo and WriteSolution (tests/golden/make_golden.py); where the
reference build exists (oracle/_ref) the tests also round-trip through its
ReadGridGeo, ReadHllcInit and WriteSolution.  Bar: bit-identical fields; file
bytes identical except the 6 padding bytes of each geo_cell_t."""
import os

import numpy as np
import pytest

import oracle
from golden_io import GOLDEN, load, mesh
from radrhd_solver_b200 import files_sys as fs
from radrhd_solver_b200.mesh import fibonacci_directions, kuhn_box

MESH_FIELDS = ("face_id_l", "face_id_r", "face_n", "face_area", "cell_faces", "cell_sign", "cell_volume",
               "cell_center")
HAVE_REF = oracle.have_ref("hydro_ideal_5_3")
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) absent")


def _same_mesh(a, b):
    for k in MESH_FIELDS:
        x, y = np.asarray(getattr(a, k) if not isinstance(a, dict) else a[k]), np.asarray(
            getattr(b, k) if not isinstance(b, dict) else b[k])
        assert x.dtype == y.dtype and np.array_equal(x, y), k


def _cell_bytes_no_pad(path):
    raw = np.fromfile(path, np.uint8)
    return raw[:4], raw[4:].reshape(-1, 56)[:, :50]


def _box():
    return kuhn_box(3, 2, 2, jitter=0.2, seed=4, bc_codes=(-1, -2, -3, -4, -5, -6), inflow_radius=0.3,
                    inflow_code=-7)


def test_record_layouts():
    assert (fs.GEO_FACE.itemsize, fs.GEO_CELL.itemsize, fs.FLUX.itemsize) == (40, 56, 40)
    if HAVE_REF:
        assert oracle.loader.ref_record_sizes() == (40, 56, 40)


def test_read_reference_written_golden_files():
    g = load("files_sys")
    d = os.path.join(GOLDEN, "files_sys")
    m, flags = fs.read_grid_geo(os.path.join(d, fs.F_GEO_FACES), os.path.join(d, fs.F_GEO_CELLS), with_flags=True)
    _same_mesh(m, mesh(g))
    assert (m.face_id_r < 0).any() and set(np.unique(m.face_id_r[m.face_id_r < 0])) <= {-1, -2, -3, -4, -5, -6, -7}
    assert -7 in m.face_id_r
    # the records the reference wrote carry its default flags
    assert (flags.face_is_regular == 1).all() and not flags.face_id_l_node.any() and not flags.cell_is_bound.any()
    assert m.h_min == fs.mesh_h_min(mesh(g)) and m.h_min > 0
    sol = fs.read_solution(os.path.join(d, "Solve0"))
    W = g["W"]
    assert set(sol) == {"density", "pressure", "velocity"}
    assert np.array_equal(sol["density"], W[:, 0]) and np.array_equal(sol["pressure"], W[:, 4])
    assert np.array_equal(sol["velocity"], W[:, 1:4])


def test_write_matches_reference_written_golden_files(tmp_path):
    g = load("files_sys")
    d = os.path.join(GOLDEN, "files_sys")
    fs.write_grid_geo(mesh(g), str(tmp_path / fs.F_GEO_FACES), str(tmp_path / fs.F_GEO_CELLS))
    assert (tmp_path / fs.F_GEO_FACES).read_bytes() == open(os.path.join(d, fs.F_GEO_FACES), "rb").read()
    h0, c0 = _cell_bytes_no_pad(str(tmp_path / fs.F_GEO_CELLS))
    h1, c1 = _cell_bytes_no_pad(os.path.join(d, fs.F_GEO_CELLS))
    assert np.array_equal(h0, h1) and np.array_equal(c0, c1)
    paths = fs.write_solution(str(tmp_path / "Solve0"), W=g["W"])
    assert sorted(os.path.basename(p) for p in paths) == ["density.bin", "pressure.bin", "velocity.bin"]
    for p in paths:
        assert open(p, "rb").read() == open(os.path.join(d, "Solve0", os.path.basename(p)), "rb").read()


@needs_ref
def test_geo_round_trip_through_reference(tmp_path):
    m = _box()
    flags = fs.GeoFlags.defaults(m.n_faces, m.n_cells)
    rng = np.random.default_rng(3)
    flags.face_id_l_node[:] = rng.integers(0, 64, m.n_faces)
    flags.face_id_r_node[:] = rng.integers(0, 64, m.n_faces)
    flags.face_is_regular[:] = rng.integers(0, 2, m.n_faces)
    flags.cell_node[:] = rng.integers(0, 64, m.n_cells)
    flags.cell_is_bound[:] = rng.integers(0, 4, m.n_cells)
    ff, cf = str(tmp_path / "f.bin"), str(tmp_path / "c.bin")
    fs.write_grid_geo(m, ff, cf, flags)
    back = oracle.loader.ref_read_geo(ff, cf)  # the reference's ReadGridGeo
    _same_mesh(back, m)
    m2, fl2 = fs.read_grid_geo(ff, cf, with_flags=True)
    _same_mesh(m2, m)
    for k in ("face_id_l_node", "face_id_r_node", "face_is_regular", "cell_node", "cell_is_bound"):
        assert np.array_equal(getattr(fl2, k), getattr(flags, k)), k
    # and the other way: the reference's WriteGridGeo, read here
    h = oracle.HydroRef(m, "hydro_ideal_5_3")
    rf, rc = str(tmp_path / "rf.bin"), str(tmp_path / "rc.bin")
    assert h.write_geo(rf, rc) == 0
    h.close()
    _same_mesh(fs.read_grid_geo(rf, rc), m)


@needs_ref
def test_hllc_init_and_solution_through_reference(tmp_path):
    m = kuhn_box(3, 2, 2, jitter=0.2, seed=4)  # transmissive sides: codes the reference's step handles
    rng = np.random.default_rng(5)
    W = np.stack([10 ** rng.uniform(-1, 1, m.n_cells), *rng.uniform(-.5, .5, (3, m.n_cells)),
                  10 ** rng.uniform(-3, 0, m.n_cells)], 1)
    p = str(tmp_path / fs.F_INIT_HLLC)
    fs.write_hllc_init(p, W)
    assert np.array_equal(oracle.loader.ref_read_hllc_init(p), W)
    assert np.array_equal(fs.read_hllc_init(p), W)
    W, U = oracle.ref_p2c(W, "hydro_ideal_5_3")
    h = oracle.HydroRef(m, "hydro_ideal_5_3")
    h.set_state(W, U)
    h.step(0.2 * m.h_min, 1)
    Wr, _ = h.get_state()
    assert h.write_solution(str(tmp_path / "ref")) == 0
    h.close()
    fs.write_solution(str(tmp_path / "ours"), W=Wr)
    for name in ("density.bin", "pressure.bin", "velocity.bin"):
        assert (tmp_path / "ours" / name).read_bytes() == (tmp_path / "ref" / name).read_bytes(), name


def test_radiation_solution_files(tmp_path):
    rng = np.random.default_rng(6)
    N, G, M = 7, 2, 5
    I = rng.uniform(size=(N * G, M))
    E, F, T = rng.uniform(size=N), rng.uniform(size=(N, 3)), rng.uniform(size=(N, 3, 3))
    W = rng.uniform(size=(N, 5))
    fs.write_solution(str(tmp_path), W=W, I=I, energy=E, stream=F, impuls=T)
    s = fs.read_solution(str(tmp_path))
    # GetCellDataBySelectedDirection: element j * M + 0 of the row-major array, j < N
    assert np.array_equal(s["Illum"], I.reshape(-1)[np.arange(N) * M])
    assert np.array_equal(s["energy"], E) and np.array_equal(s["stream"], F) and np.array_equal(s["impuls"], T)
    raw = (tmp_path / "Illum.bin").read_bytes()
    assert len(raw) == 4 + 8 * N and int(np.frombuffer(raw[:4], "<i4")[0]) == N


def test_errors(tmp_path):
    m = _box()
    ff, cf = str(tmp_path / "f.bin"), str(tmp_path / "c.bin")
    fs.write_grid_geo(m, ff, cf)
    raw = open(ff, "rb").read()
    open(ff, "wb").write(raw[:-8])  # truncated last record
    with pytest.raises(OSError):
        fs.read_grid_geo(ff, cf)
    open(ff, "wb").write(raw[:2])  # no count
    with pytest.raises(OSError):
        fs.read_grid_geo(ff, cf)
    bad = fs.encode_faces(m.face_id_l, m.face_id_r, m.face_n, m.face_area)
    bad["w0"][0] = m.n_cells  # id_l past the last cell
    fs._write_records(ff, m.n_faces, bad)
    with pytest.raises(ValueError):
        fs.read_grid_geo(ff, cf)
    with pytest.raises(ValueError):
        fs.encode_faces([1 << 25], [0], np.zeros((1, 3)), [1.0])
    with pytest.raises(ValueError):
        fs.encode_faces([0], [-(1 << 25) - 1], np.zeros((1, 3)), [1.0])
    # empty files are valid
    e = fs.read_simple(str(_empty(tmp_path)))
    assert e.shape == (0,)


def _empty(tmp_path):
    p = tmp_path / "empty.bin"
    p.write_bytes(np.int32(0).tobytes())
    return p


def test_sphere_directions(tmp_path):
    d = fibonacci_directions(37)
    p = str(tmp_path / "grid_direction.txt")
    fs.write_sphere_directions(p, d)
    r = fs.read_sphere_directions(p)
    assert np.array_equal(r.dirs, d.dirs) and np.array_equal(r.areas, d.areas) and r.full_area == d.full_area
    if HAVE_REF:  # the reference's ReadSphereDirectionCartesian reads the same doubles
        dirs, areas, full = oracle.loader.ref_read_sphere_directions(p)
        assert np.array_equal(dirs, d.dirs) and np.array_equal(areas, d.areas) and full == d.full_area
    open(p, "w").write("3\n1 0 0 1\n")
    with pytest.raises(OSError):
        fs.read_sphere_directions(p)
