"""GPU tests of device-side parcel initialisation, the ParaView writer and restart files.

  - st_init_parcels: the parcels generated on the device equal the oracle's (the same
    counter-based generator compiled for the host) bit for bit, in every precision;
  - st_write_vtu / st_write_pvd: the file parses as VTK XML, and its appended arrays hold
    exactly the parcel state of st_get_parcels;
  - st_save_state / st_load_state: a run saved after some steps and continued in a new
    handle gives the same parcels, cells and source, bit for bit, as the uninterrupted run
    (cuboid and tet meshes)."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

L = workload.L_BOX


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_device_init_matches_oracle(prec):
    N, nc, n = 20, 3, 30000
    prm = st.params(precision=prec, n_clouds=nc, sort_interval=5)
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, L)) as h:
        for c in range(nc):
            h.init_parcels(n + c, 1234, 5e-6, 5e-5, cloud=c)
        for c in range(nc):
            xyz, uvw, d = h.get_parcels(c)
            ox, od = oracle.init_parcels(4 if prec == "fp32" else 8, 1234, c, nc, n + c, N,
                                         0.0, L, 5e-6, 5e-5)
            vt = np.float64 if prec == "fp64" else np.float32
            assert np.array_equal(xyz, ox)
            assert np.array_equal(d, od.astype(vt).astype(np.float64))
            assert (uvw == 0).all()
            cells = h.get_cells(c)
            assert (cells >= 0).all() and (cells < N ** 3).all()


def test_vtu_and_pvd(tmp_path):
    N, n = 12, 5000
    prm = st.params(precision="mixed", drag_model="schiller_naumann", n_substeps=1,
                    mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P)
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, L)) as h:
        h.init_parcels(n, 9, 5e-6, 5e-5)
        h.set_fluid_velocity(workload.tgv_field(N))
        h.step(workload.DT)
        p = str(tmp_path / "parcels_0.vtu")
        h.write_vtu(p)
        xyz, uvw, d = h.get_parcels()
    raw = open(p, "rb").read()
    start = raw.index(b"<AppendedData encoding=\"raw\">")
    xml_head = raw[:start].decode() + "</VTKFile>"
    root = ET.fromstring(xml_head)
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfPoints")) == n
    data = raw[raw.index(b"_", start) + 1:]
    arrays = {}
    for da in root.iter("DataArray"):
        off = int(da.get("offset"))
        size = int(np.frombuffer(data[off:off + 8], dtype="<u8")[0])
        dt = {"Float64": "<f8", "Int64": "<i8", "UInt8": "u1"}[da.get("type")]
        arrays[da.get("Name")] = np.frombuffer(data[off + 8:off + 8 + size], dtype=dt)
    assert np.array_equal(arrays["Points"].reshape(n, 3), xyz.T)
    assert np.array_equal(arrays["U"].reshape(n, 3), uvw.T)
    assert np.array_equal(arrays["d"], d)
    assert np.array_equal(arrays["connectivity"], np.arange(n))
    assert np.array_equal(arrays["offsets"], np.arange(1, n + 1))
    assert (arrays["types"] == 1).all()
    pvd = str(tmp_path / "parcels.pvd")
    st.write_pvd(pvd, [0.0, 1e-4], ["parcels_0.vtu", "parcels_1.vtu"])
    ds = ET.parse(pvd).getroot().findall("Collection/DataSet")
    assert [d_.get("file") for d_ in ds] == ["parcels_0.vtu", "parcels_1.vtu"]
    assert [float(d_.get("timestep")) for d_ in ds] == [0.0, 1e-4]


def _hex_run(prm, N, xyz, uvw, d, U, fs, save_at=None, path=None, load=None):
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, L)) as h:
        if load:
            h.load_state(load)
        else:
            h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k, f in enumerate(fs):
            if save_at is not None and k == save_at:
                h.save_state(path)
            h.step(workload.DT, f)
        h.synchronize()
        return h.get_parcels()[0], h.get_cells(), h.get_source(0)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_restart_continues_bit_for_bit(tmp_path, prec):
    N, n = 16, 20000
    prm = st.params(precision=prec, drag_model="schiller_naumann", n_substeps=1,
                    sort_interval=3, mu_c=workload.MU_F, rho_c=workload.RHO_F,
                    rho_d=workload.RHO_P)
    xyz, uvw, d = workload.parcels(n, 4)
    U = workload.tgv_field(N, dtype=np.float64 if prec == "fp64" else np.float32)
    fs = [workload.fluid_scale(k) for k in range(8)]
    path = str(tmp_path / "state.bin")
    full = _hex_run(prm, N, xyz, uvw, d, U, fs, save_at=5, path=path)
    cont = _hex_run(prm, N, None, None, None, U, fs[5:], load=path)
    for a, b in zip(full, cont):
        assert np.array_equal(a, b)


def test_restart_on_tet_mesh(tmp_path):
    n_hex, m = 6, 8000
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n_hex, L, 0.15, 1)
    xyz, _, d = workload.parcels(m, 8)
    uvw = np.random.default_rng(8).normal(0, 3.0, (3, m)).astype(np.float32).astype(np.float64)
    U = workload.tgv_at(workload.tet_centroids(verts, tets), U0=3.0)
    hint = workload.tet_hints(xyz, hex_ijk, n_hex, L)
    prm = st.params(precision="mixed", drag_model="schiller_naumann", n_substeps=1,
                    sort_interval=2, mu_c=workload.MU_F, rho_c=workload.RHO_F,
                    rho_d=workload.RHO_P)
    desc = st.tet_mesh_desc(verts, tets, nbr, 0.0, L)
    path = str(tmp_path / "tet_state.bin")
    fs = [workload.fluid_scale(k) for k in range(6)]

    def run(load):
        with st.ParcelTracker(prm, desc) as h:
            if load:
                h.load_state(path)
                steps = fs[3:]
            else:
                h.set_parcels(xyz, uvw, d, hint=hint)
                steps = fs
            h.set_fluid_velocity(U)
            for k, f in enumerate(steps):
                if not load and k == 3:
                    h.save_state(path)
                h.step(1e-3, f)
            h.synchronize()
            return h.get_parcels()[0], h.get_cells(), h.get_source(0)

    full = run(False)
    cont = run(True)
    for a, b in zip(full, cont):
        assert np.array_equal(a, b)


def test_load_state_rejects_other_handles(tmp_path):
    prm = st.params(precision="mixed")
    path = str(tmp_path / "s.bin")
    with st.ParcelTracker(prm, st.mesh_desc(8, 0.0, L)) as h:
        h.init_parcels(100, 1, 5e-6, 5e-5)
        h.save_state(path)
    with st.ParcelTracker(st.params(precision="fp64"), st.mesh_desc(8, 0.0, L)) as h2:
        with pytest.raises(st.ScaleTrackError):
            h2.load_state(path)
    with open(str(tmp_path / "junk.bin"), "wb") as f:
        f.write(b"nonsense")
    with st.ParcelTracker(prm, st.mesh_desc(8, 0.0, L)) as h3:
        with pytest.raises(st.ScaleTrackError):
            h3.load_state(str(tmp_path / "junk.bin"))


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_append_parcels_continues_like_the_oracle(prec):
    """Injection: parcels appended after two steps (the buffers grow on the device) step on
    with the others exactly as the oracle steps the combined set."""
    N, n, m = 12, 3000, 2500
    xyz, uvw, d = workload.parcels(n + m, 19)
    vt = np.float64 if prec == "fp64" else np.float32
    U = workload.tgv_field(N, dtype=vt)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision=prec, n_substeps=1,
                    sort_interval=2)
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, L)) as h:
        h.set_parcels(xyz[:, :n], uvw[:, :n], d[:n])
        h.set_fluid_velocity(U)
        h.step(workload.DT)
        h.step(workload.DT)
        h.append_parcels(xyz[:, n:], uvw[:, n:], d[n:])
        assert h.num_parcels() == n + m
        h.step(workload.DT)
        h.step(workload.DT)
        h.synchronize()
        gx, gv, _ = h.get_parcels()
        gc = h.get_cells()
        gs = h.get_source(0)
    cfg = oracle.make_cfg(N, 0.0, L, workload.MU_F, workload.RHO_F, workload.RHO_P,
                          drag="sn_explicit", precision=prec, n_substeps=1,
                          quant_limbs=2 if prec == "fp64" else 1)
    U64 = U.astype(np.float64)
    r1 = oracle.run(cfg, xyz[:, :n], uvw[:, :n], d[:n], U64, 2, workload.DT)
    x2 = np.concatenate([r1["xyz"], xyz[:, n:]], axis=1)
    v2 = np.concatenate([r1["uvw"], uvw[:, n:].astype(vt).astype(np.float64)], axis=1)
    r2 = oracle.run(cfg, x2, v2, d, U64, 2, workload.DT)
    assert np.array_equal(gx, r2["xyz"]) and np.array_equal(gv, r2["uvw"])
    assert np.array_equal(gc, r2["cells"])
    assert np.array_equal(gs, r2["src_quant"])


def test_load_state_checks_the_whole_file_before_changing_the_handle(tmp_path):
    """A truncated file, or one with an impossible fixed-point scale, is rejected and the
    handle keeps its parcels."""
    prm = st.params(precision="mixed")
    path = str(tmp_path / "s.bin")
    with st.ParcelTracker(prm, st.mesh_desc(8, 0.0, L)) as h:
        h.init_parcels(100, 1, 5e-6, 5e-5)
        h.save_state(path)
    raw = open(path, "rb").read()
    hdr = 8 + 16 + 8 + 8 + 8 + 8                  # magic, 4 int32, nCells, dt, steps, sched
    bad_scale = bytearray(raw)
    bad_scale[hdr:hdr + 4] = (5000).to_bytes(4, "little", signed=True)   # L
    cases = {"truncated": raw[:-12], "bad_scale": bytes(bad_scale)}
    for name, blob in cases.items():
        p = str(tmp_path / (name + ".bin"))
        with open(p, "wb") as f:
            f.write(blob)
        with st.ParcelTracker(prm, st.mesh_desc(8, 0.0, L)) as h2:
            h2.init_parcels(37, 2, 5e-6, 5e-5)
            before = h2.get_parcels()
            with pytest.raises(st.ScaleTrackError) as ei:
                h2.load_state(p)
            assert ei.value.code == st.ST_ERR_INVALID_ARGUMENT, name
            after = h2.get_parcels()
            for a, b in zip(before, after):
                assert np.array_equal(a, b), name
