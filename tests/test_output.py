"""VTK snapshot files and collections (host side of output.py; no GPU)."""
import numpy as np
import pytest


def test_vtr_roundtrip_2d(pkg, tmp_path):
    rng = np.random.default_rng(0)
    rho = rng.random((5, 7))
    ux, uy = rng.random((2, 5, 7)).astype(np.float32)
    p = pkg.output.write_vtr(tmp_path / "snap", 7, 5, None, 0.5, {"rho": rho, "velocity": (ux, uy)})
    assert p.suffix == ".vtr"
    d = pkg.output.read_vtr(p)
    assert np.array_equal(d["rho"], rho.reshape(-1))
    v = d["velocity"]
    assert v.shape == (35, 3) and v.dtype == np.float32
    assert np.array_equal(v[:, 0], ux.reshape(-1)) and np.array_equal(v[:, 1], uy.reshape(-1))
    assert np.all(v[:, 2] == 0)
    assert np.array_equal(d["x_coordinates"], np.arange(8) * 0.5)
    assert np.array_equal(d["y_coordinates"], np.arange(6) * 0.5)
    text = p.read_bytes()[:400].decode(errors="ignore")
    assert 'WholeExtent="0 7 0 5 0 0"' in text and "<CellData>" in text


def test_vtr_roundtrip_3d_and_half(pkg, tmp_path):
    rng = np.random.default_rng(1)
    a = rng.random((3, 4, 5)).astype(np.float16)
    comps = tuple(rng.random((3, 4, 5)) for _ in range(3))
    p = pkg.output.write_vtr(tmp_path / "s3", 5, 4, 3, 1.0, {"T": a, "u": comps})
    d = pkg.output.read_vtr(p)
    assert np.array_equal(d["T"], a.astype(np.float32).reshape(-1))
    for n in range(3):
        assert np.array_equal(d["u"][:, n], comps[n].reshape(-1))
    assert d["z_coordinates"].shape == (4,)


def test_pvd_collection(pkg, tmp_path):
    import xml.etree.ElementTree as ET
    s = pkg.output.VTKSeries(tmp_path, 4, 3, name="run")
    for step in (10, 20):
        s(step, step * 0.1, {"rho": np.ones((3, 4))})
    s.close()
    root = ET.parse(tmp_path / "run.pvd").getroot()
    ds = root.find("Collection").findall("DataSet")
    assert [d.get("file") for d in ds] == ["snapshot_0000010.vtr", "snapshot_0000020.vtr"]
    assert [float(d.get("timestep")) for d in ds] == pytest.approx([1.0, 2.0])
    assert (tmp_path / "snapshot_0000020.vtr").exists()
