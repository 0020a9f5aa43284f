"""The C ABI library on the host: loads, exports every entry point declared
in include/hipft_gpu.h, reads the reference's HDF5 maps, and rejects bad
arguments before touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "hipft_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*\*?\s*(hipft_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    import hipft_b200 as H
    L = H.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert b"sm_100a" in L.hipft_gpu_version()


def test_binding_covers_header():
    from hipft_b200 import gpu
    bound = {n for n, _, _ in gpu.SIGNATURES}
    assert set(declared_functions()) <= bound


@pytest.mark.parametrize("case,shape", [("diffuse_dipole", (512, 1024)),
                                        ("diffuse_advect_atten_map_1cr", (180, 360))])
def test_h5_read_testsuite_maps(case, shape):
    import hipft_b200 as H
    p = cases.params(case)
    d, sc = H.h5_read(os.path.join(cases.input_dir(case), p["initial_map_filename"]))
    assert d.shape == shape
    assert sc[0].shape == (shape[1],) and sc[1].shape == (shape[0],)
    assert abs(sc[0][0]) < 1e-6 and abs(sc[0][-1] - 2 * np.pi) < 1e-5
    assert abs(sc[1][0]) < 1e-6 and abs(sc[1][-1] - np.pi) < 1e-5
    assert np.isfinite(d).all() and np.abs(d).max() > 100.0


def test_h5_read_rejects_non_hdf5(tmp_path):
    import hipft_b200 as H
    bad = tmp_path / "x.h5"
    bad.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(H.HipftError) as e:
        H.h5_read(str(bad))
    assert e.value.code == 6
    with pytest.raises(H.HipftError):
        H.h5_read(str(tmp_path / "missing.h5"))


def test_create_rejects_bad_arguments():
    from hipft_b200 import gpu
    L = gpu.lib()
    h = ctypes.c_void_p()
    t = np.linspace(0, np.pi, 3)
    p = np.linspace(0, 2 * np.pi, 8)
    g = gpu.Grid(3, 8, 1, 0, t.ctypes.data_as(gpu.DPTR), p.ctypes.data_as(gpu.DPTR))  # ntm too small
    prm = gpu.Params()
    assert L.hipft_gpu_create(ctypes.byref(g), ctypes.byref(prm), ctypes.byref(h)) == gpu.HIPFT_EINVAL
    assert L.hipft_gpu_create(None, ctypes.byref(prm), ctypes.byref(h)) == gpu.HIPFT_EINVAL
    t = np.linspace(0, np.pi, 16)
    g = gpu.Grid(16, 8, 1, 0, t.ctypes.data_as(gpu.DPTR), p.ctypes.data_as(gpu.DPTR))
    prm.advance_diffusion = 1  # without diffusion constants
    prm.diffusion_num_method = 3
    assert L.hipft_gpu_create(ctypes.byref(g), ctypes.byref(prm), ctypes.byref(h)) == gpu.HIPFT_EINVAL
    prm.advance_diffusion = 0
    prm.advance_flow = 1
    prm.flow_num_method = 7
    assert L.hipft_gpu_create(ctypes.byref(g), ctypes.byref(prm), ctypes.byref(h)) == gpu.HIPFT_EINVAL
    # null handles are rejected, not dereferenced
    assert L.hipft_gpu_advection_step(None, 1.0) == gpu.HIPFT_EINVAL
    assert L.hipft_gpu_destroy(None) == gpu.HIPFT_OK


def test_run_rejects_bad_namelist(tmp_path):
    import hipft_b200 as H
    nl = tmp_path / "hipft.in"
    nl.write_text("&hipft_input_parameters\n  res_nt = 2\n  res_np = 2\n/\n")
    with pytest.raises(H.HipftError) as e:
        H.run(str(nl), str(tmp_path))
    assert e.value.code == 1
    nl.write_text("&hipft_input_parameters\n  res_nt = 20\n  res_np = 40\n  no_such_variable = 3\n/\n")
    with pytest.raises(H.HipftError):
        H.run(str(nl), str(tmp_path))
    nl.write_text("&hipft_input_parameters\n  res_nt = 20\n res_np = 40\n flow_num_method = 9\n/\n")
    with pytest.raises(H.HipftError):
        H.run(str(nl), str(tmp_path))
