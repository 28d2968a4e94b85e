"""The post-processing reader with the reference's interface (ext/python/read_cruna_data.py:37-236)
on this library's snapshot container, on the CPU: files written by the library's C writer are read
back bit-exactly in plain Python, one component or all, one block image or several placed by their
global index ranges, and parameters become the reference's nested dict."""
import numpy as np
import pytest

from public_b200 import cruna
from public_b200.read_cruna_data import read_cruna_data, read_cruna_params

PARAMS = ("geom.n1 = 6\ngeom.n2 = 5\ngeom.n3 = 4\ntime.dt = 1.25e-3\ntime.nt = 100\n"
          "material.gamma = 1.4\nparallelism.i1 = 1\nparallelism.i2 = 1\nparallelism.i3 = 1\n")


def _state(seed, shape=(6, 5, 4, 5)):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(shape))


def test_single_image_all_components_and_one(tmp_path):
    q = _state(0)
    name = cruna.io_fname(str(tmp_path), "data_direct_snapshot", ns=1, nt=100)
    cruna.write_snapshot(name, q, PARAMS)
    data, params = read_cruna_data(name)
    assert data.shape == (6, 5, 4, 5)
    assert np.array_equal(data.view(np.uint64), q.view(np.uint64))
    assert params["geom"]["n1"] == 6.0 and params["time"]["dt"] == 1.25e-3
    p4, _ = read_cruna_data(name, component=4)
    assert p4.shape == (6, 5, 4) and np.array_equal(p4, q[..., 4])
    again, same = read_cruna_data(name, read_params=[False, params])
    assert same is params and np.array_equal(again, q)


def test_block_images_are_placed_by_their_global_index_ranges(tmp_path):
    q = _state(1, (8, 5, 4, 5))
    w = str(tmp_path)
    base = ("geom.n1 = 8\ngeom.n2 = 5\ngeom.n3 = 4\nparallelism.i1 = 2\nparallelism.i2 = 1\n"
            "parallelism.i3 = 1\n")
    for img, (lo, hi) in enumerate(((1, 3), (4, 8)), start=1):
        rng = (f"geom.xi10i = {lo}\ngeom.xi11i = {hi}\ngeom.xi20i = 1\ngeom.xi21i = 5\n"
               f"geom.xi30i = 1\ngeom.xi31i = 4\n")
        name = f"{w}/data_direct_snapshot__01_{img:05d}_01_0000007.bin"
        cruna.write_snapshot(name, np.asfortranarray(q[lo - 1:hi]), base + rng)
    data, params = read_cruna_data(f"{w}/data_direct_snapshot__01_00001_01_0000007.bin")
    assert np.array_equal(data, q)
    one, _ = read_cruna_data(f"{w}/data_direct_snapshot__01_00001_01_0000007.bin", images=[2], component=0)
    assert np.array_equal(one[3:8], q[3:8, ..., 0]) and not one[:3].any()


def test_several_images_without_index_ranges_are_refused(tmp_path):
    w = str(tmp_path)
    for img in (1, 2):
        cruna.write_snapshot(f"{w}/data_direct_snapshot__01_{img:05d}_01_0000001.bin", _state(img), PARAMS)
    with pytest.raises(NotImplementedError):
        read_cruna_data(f"{w}/data_direct_snapshot__01_00001_01_0000001.bin", images=[1, 2])


def test_ascii_parameter_file(tmp_path):
    path = tmp_path / "parameter.dat"
    path.write_text("% a comment line\n"
                    "geom.n1 = 64       % points in x\n"
                    "sponge.amplitude = 1.0;2.0;3.0\n"
                    "io.workdir = ./run\n"
                    "\n"
                    "bc.zone.type = 201\n")
    p = read_cruna_params(str(path))
    assert p["geom"]["n1"] == 64.0
    assert p["sponge"]["amplitude"] == [1.0, 2.0, 3.0]
    assert p["io"]["workdir"] == "./run"
    assert p["bc"]["zone"]["type"] == 201.0


def test_foreign_and_truncated_files_are_rejected(tmp_path):
    bad = tmp_path / "data_direct_snapshot__01_00001_01_0000001.bin"
    bad.write_bytes(b"\0" * 100)
    with pytest.raises(ValueError):
        read_cruna_data(str(bad))
    good = str(tmp_path / "data_direct_snapshot__01_00001_01_0000002.bin")
    cruna.write_snapshot(good, _state(3), PARAMS)
    raw = open(good, "rb").read()
    open(good, "wb").write(raw[:-16])
    with pytest.raises(ValueError):
        read_cruna_data(good)
