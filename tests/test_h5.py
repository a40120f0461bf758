"""The package's HDF5 writer (output.h5) against its structural reader: the
tree, every dataset's type, size and values, names in order, and the file's
end-of-file address.  No HDF5 library exists beside the package to read the
files independently; the layout written is the subset of the HDF5 format the
reference's output.h5 uses (superblock 0, version-1 object headers, symbol-table
groups, contiguous 1-D datasets of double, int32 and uint8)."""
import os

import numpy as np
import pytest


def test_roundtrip_tree(pkg, tmp_path):
    h5 = pkg.h5
    t = h5.H5Tree()
    j = t.group("json")
    j.write("tb_file", "hBN_gap7.25eV_a2.5A")
    j.write("coulomb", 1)
    j.write("grid", np.array([50, 50, 1], dtype=np.int32))
    j.write("dt", 0.1)
    j.group("laser0").write("intensity", 1e10)
    rng = np.random.default_rng(0)
    z = rng.normal(size=(7, 3, 3)) + 1j * rng.normal(size=(7, 3, 3))
    t.group("DensityMatrix_k").group("0").group("0").write("local", z)
    tg = t.group("time_au")
    for i in range(300):  # more members than one symbol-table node holds
        tg.write(str(i), 0.5 * i)
    path = os.path.join(str(tmp_path), "output.h5")
    t.save(path)
    got = h5.read_h5(path)
    assert sorted(got) == ["DensityMatrix_k", "json", "time_au"]
    assert bytes(got["json"]["tb_file"]).decode() == "hBN_gap7.25eV_a2.5A"
    assert got["json"]["tb_file"].dtype == np.uint8
    assert got["json"]["coulomb"].dtype == np.int32 and got["json"]["coulomb"].tolist() == [1]
    assert got["json"]["grid"].tolist() == [50, 50, 1]
    assert got["json"]["dt"].dtype == np.float64 and got["json"]["dt"].tolist() == [0.1]
    assert got["json"]["laser0"]["intensity"].tolist() == [1e10]
    local = got["DensityMatrix_k"]["0"]["0"]["local"]
    assert local.dtype == np.float64 and local.size == 2 * z.size
    assert np.array_equal(local.view(np.complex128).reshape(z.shape), z)
    assert len(got["time_au"]) == 300
    assert all(got["time_au"][str(i)].tolist() == [0.5 * i] for i in range(300))
    with open(path, "rb") as f:
        head = f.read(8)
    assert head == b"\x89HDF\r\n\x1a\n"


def test_refuses_bad_input(pkg):
    t = pkg.h5.H5Tree()
    t.write("a", 1.0)
    with pytest.raises(ValueError):
        t.write("a", 2.0)
    with pytest.raises(ValueError):
        t.group("a")
    with pytest.raises(ValueError):
        t.write("empty", np.zeros(0))


def test_corruption_is_detected(pkg, tmp_path):
    t = pkg.h5.H5Tree()
    t.write("x", np.arange(5.0))
    path = os.path.join(str(tmp_path), "c.h5")
    t.save(path)
    with open(path, "rb") as f:
        b = bytearray(f.read())
    with open(path, "wb") as f:
        f.write(bytes(b[:-8]))  # truncated: the end-of-file address no longer matches
    with pytest.raises(ValueError):
        pkg.h5.read_h5(path)
