"""The HDF5 map writer (hipft_h5_write, restating wrh5 src/hipft.f90:6155-6351).

CPU tests: values and scales survive a write/read round trip (float64
exactly, float32 as the reference's REAL(x, REAL32) conversion), and the file
holds what the HDF5 library expects of such a map: "Data" plus "dim1".."dimN"
in a symbol-table root group, each scale marked CLASS = DIMENSION_SCALE with
NAME = dimN and a REFERENCE_LIST back to "Data", and "Data"'s
DIMENSION_LIST / DIMENSION_LABELS pointing at the scales.
"""
import numpy as np
import pytest

import h5_struct


def _roundtrip(tmp_path, shape, single):
    import hipft_b200 as H
    rng = np.random.default_rng(len(shape) + 10 * single)
    data = rng.normal(size=shape) * 1e3
    scales = [np.sort(rng.uniform(0, 7, size=n)) for n in reversed(shape)]
    path = str(tmp_path / "m.h5")
    H.h5_write(path, data, scales, single_precision=single)
    back, sc = H.h5_read(path)
    conv = (lambda a: a.astype(np.float32).astype(np.float64)) if single else (lambda a: a)
    assert back.shape == data.shape
    assert np.array_equal(back, conv(data))
    for a, b in zip(sc, scales):
        assert np.array_equal(a, conv(b))
    return path, data, scales


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("shape", [(9,), (17, 33), (3, 17, 33)])
def test_h5_write_roundtrip(tmp_path, shape, single):
    _roundtrip(tmp_path, shape, single)


@pytest.mark.parametrize("shape", [(17, 33), (4, 17, 33)])
def test_h5_write_structure(tmp_path, shape):
    path, data, scales = _roundtrip(tmp_path, shape, True)
    f = h5_struct.H5Struct(path)
    nd = len(shape)
    names = ["Data"] + [f"dim{i + 1}" for i in range(nd)]
    assert sorted(f.objects) == names
    # B-tree keys bracket the names of its one symbol node
    assert f.keys == [0, 8 * (1 + nd)]
    assert f.name_at(f.keys[-1]) == names[-1]
    assert f.eof == len(f.b)
    d = f.dataset("Data", strict=True)
    assert d["dims"] == list(shape) and d["class"] == 1 and d["elsize"] == 4
    assert d["size"] == data.size * 4
    raw = np.frombuffer(f.b, dtype="<f4", count=data.size, offset=d["addr"])
    assert np.array_equal(raw.reshape(shape), data.astype(np.float32))
    dl = d["attrs"]["DIMENSION_LIST"]
    assert [r[0] for r in dl] == [f.objects[f"dim{i + 1}"] for i in range(nd)]
    assert d["attrs"]["DIMENSION_LABELS"] == [f"dim{i + 1}" for i in range(nd)]
    for i in range(nd):
        s = f.dataset(f"dim{i + 1}", strict=True)
        assert s["dims"] == [len(scales[i])]
        assert s["attrs"]["CLASS"] == "DIMENSION_SCALE"
        assert s["attrs"]["NAME"] == f"dim{i + 1}"
        assert s["attrs"]["REFERENCE_LIST"] == [(f.objects["Data"], i)]


def test_h5_write_float64_layout(tmp_path):
    path, data, _ = _roundtrip(tmp_path, (5, 7), False)
    f = h5_struct.H5Struct(path)
    d = f.dataset("Data")
    assert d["elsize"] == 8
    raw = np.frombuffer(f.b, dtype="<f8", count=data.size, offset=d["addr"])
    assert np.array_equal(raw.reshape(data.shape), data)


def test_h5_write_rejects_bad_arguments(tmp_path):
    import hipft_b200 as H
    from hipft_b200 import gpu
    with pytest.raises(ValueError):
        H.h5_write(str(tmp_path / "x.h5"), np.zeros((2, 3)), [np.zeros(3)])
    with pytest.raises(gpu.HipftError) as e:
        H.h5_write(str(tmp_path / "no_such_dir" / "x.h5"), np.zeros((2, 3)), [np.zeros(3), np.zeros(2)])
    assert e.value.code == gpu.HIPFT_EIO


def test_reference_map_has_the_structure_the_writer_emulates():
    """The testsuite's input map, written by the HDF5 library, holds the same
    objects and attribute set as the writer's output (its DIMENSION_LIST uses
    the same entry-c-is-dim<c+1> convention)."""
    import os
    import cases
    path = os.path.join(cases.input_dir("diffuse_dipole"), "br_input.h5")
    f = h5_struct.H5Struct(path)
    assert sorted(f.objects) == ["Data", "dim1", "dim2"]
    d = f.dataset("Data")
    assert set(d["attrs"]) == {"DIMENSION_LIST", "DIMENSION_LABELS"}
    assert d["attrs"]["DIMENSION_LABELS"] == ["dim1", "dim2"]
    assert [r[0] for r in d["attrs"]["DIMENSION_LIST"]] == [f.objects["dim1"], f.objects["dim2"]]
    for i in range(2):
        s = f.dataset(f"dim{i + 1}")
        assert set(s["attrs"]) == {"CLASS", "NAME", "REFERENCE_LIST"}
        assert s["attrs"]["CLASS"] == "DIMENSION_SCALE" and s["attrs"]["NAME"] == f"dim{i + 1}"
        assert s["attrs"]["REFERENCE_LIST"] == [(f.objects["Data"], i)]
