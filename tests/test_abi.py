"""CPU tests of the C ABI: the library builds for sm_100a, loads, exports every entry point
declared in include/scaletrack.h, validates arguments and refuses to run without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import scaletrack as st

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    with open(os.path.join(ROOT, "include", "scaletrack.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"ST_API[^;(]*?\b(st_\w+)\(", text)))


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_loads_and_exports_header_symbols():
    L = st.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(st.EXPORTS) == syms
    assert b"sm_100a" in L.st_version()


def test_only_declared_symbols_are_exported():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", st.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = sorted(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert exported == header_symbols()


def test_params_default_is_reference_setup():
    p = st.params()
    assert (p.mu_c, p.rho_c, p.rho_d) == (1e-3, 1e3, 1.0)  # setup.jl:12-14
    assert p.n_substeps == 10                                # A:1260
    assert p.precision == 0 and p.drag_model == 0 and p.n_clouds == 1
    assert p.drag_multiplier == 1.0 and p.diameter_scale == 1.0


@pytest.mark.parametrize("kw,mesh", [
    (dict(precision=7), (8, 0, 1)),
    (dict(n_substeps=0), (8, 0, 1)),
    (dict(n_clouds=0), (8, 0, 1)),
    (dict(mu_c=-1.0), (8, 0, 1)),
    (dict(block_size=100), (8, 0, 1)),
    (dict(), (0, 0, 1)),
    (dict(), (8, 1, 1)),
])
def test_create_rejects_bad_arguments(kw, mesh):
    with pytest.raises(st.ScaleTrackError) as e:
        st.ParcelTracker(st.params(**kw), st.mesh_desc(*mesh))
    assert e.value.code == st.ST_ERR_INVALID_ARGUMENT
    assert st.last_error()


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    with pytest.raises(st.ScaleTrackError) as e:
        st.ParcelTracker(st.params(), st.mesh_desc(8, 0.0, 1.0))
    assert e.value.code == st.ST_ERR_CUDA
    assert "no CUDA device" in str(e.value)


def test_shims_before_setup_fail_cleanly():
    L = st.lib()
    L.st_finalize()
    assert L.st_allocate_array(b"U", 512, 3, 4) is None
    assert "before st_setup" in st.last_error()
    assert L.st_evolve_cloud(ctypes.c_double(1e-3)) == st.ST_ERR_NOT_INITIALISED


def test_null_handle_is_rejected():
    L = st.lib()
    assert L.st_step(None, 1e-3, 1.0) == st.ST_ERR_INVALID_ARGUMENT
    assert L.st_synchronize(None) == st.ST_ERR_INVALID_ARGUMENT
    assert L.st_num_parcels(None, 0) == -1
    assert L.st_launch_count(None) == -1


def test_pvd_collection_written_on_the_host(tmp_path):
    """st_write_pvd is host-only: the collection lists every dump with its time."""
    import xml.etree.ElementTree as ET
    path = str(tmp_path / "c.pvd")
    st.write_pvd(path, [0.0, 2.5e-4, 5e-4], ["a.vtu", "b.vtu", "c.vtu"])
    ds = ET.parse(path).getroot().findall("Collection/DataSet")
    assert [d.get("file") for d in ds] == ["a.vtu", "b.vtu", "c.vtu"]
    assert [float(d.get("timestep")) for d in ds] == [0.0, 2.5e-4, 5e-4]
    assert st.lib().st_write_pvd(None, 0, None, None) == st.ST_ERR_INVALID_ARGUMENT


def test_exchange_mode_is_validated():
    assert st.lib().st_set_exchange_mode(7) == st.ST_ERR_INVALID_ARGUMENT
    assert "exchange mode" in st.last_error()
    st.set_exchange_mode("copy")


def test_host_wrapper_rejects_malformed_tet_meshes():
    """Shape errors are raised by the Python host before anything reaches the library."""
    v = np.zeros((5, 3))
    t = np.zeros((2, 4), np.int32)
    with pytest.raises(ValueError):
        st.tet_mesh_desc(np.zeros((5, 2)), t, t, 0.0, 1.0)
    with pytest.raises(ValueError):
        st.tet_mesh_desc(v, t, np.zeros((3, 4), np.int32), 0.0, 1.0)
    d = st.tet_mesh_desc(v, t, t, 0.0, 1.0)
    assert d.n_vertices == 5 and d.n_tets == 2
