"""Snapshot and restart files on the CPU (no GPU): the reference's file names
(src/helper/io_helper.f90:11-15, 426-432), bit-exact write/read round trips of the binary container
that stands in for the reference's HDF5 store (src/io/hdf5_single.f90:659-774), the restartfile
(ns, nt) pair, and the restart arithmetic of src/main/cruna_hpc.f90:143-145."""
import os

import numpy as np
import pytest

from public_b200 import cruna


def test_file_names_follow_the_reference_scheme(tmp_path):
    w = str(tmp_path)
    assert cruna.io_fname(w, "data_direct_snapshot", ns=1, nt=100) == f"{w}/data_direct_snapshot__01_00001_01_0000100.bin"
    assert cruna.io_fname(w, "data_adjoint_snapshot", ns=3, nt=7) == f"{w}/data_adjoint_snapshot__01_00001_03_0000007.bin"
    assert cruna.io_fname(w, "data_direct", ns=2) == f"{w}/data_direct__01_00001_02.bin"
    assert cruna.io_fname(w, "restartfile") == f"{w}/restartfile.bin"
    assert cruna.io_fname("", "restartfile") == "./restartfile.bin"
    with pytest.raises(cruna.CrunaError):
        cruna.io_fname(w, "no_such_type")


def test_snapshot_round_trip_is_bit_exact(tmp_path):
    rng = np.random.default_rng(0)
    q = np.asfortranarray(rng.standard_normal((7, 5, 3, 5)) * 10.0 ** rng.integers(-300, 300, (7, 5, 3, 5)))
    path = str(tmp_path / "snap.bin")
    cruna.write_snapshot(path, q, "geom.n1 = 7\ntime.nt = 12\n")
    back, params = cruna.read_snapshot(path)
    assert back.shape == q.shape and back.flags.f_contiguous
    assert np.array_equal(back.view(np.uint64), q.view(np.uint64))
    assert "time.nt = 12" in params
    assert not os.path.exists(path + ".tmp")


def test_corrupt_or_foreign_files_are_rejected(tmp_path):
    path = tmp_path / "bad.bin"
    path.write_bytes(b"not a snapshot at all, just bytes" * 4)
    with pytest.raises(cruna.CrunaError) as e:
        cruna.read_snapshot(str(path))
    assert e.value.code == -7                        # CRUNA_ERR_IO
    good = str(tmp_path / "good.bin")
    cruna.write_snapshot(good, np.ones((4, 4, 4, 5), order="F"))
    raw = open(good, "rb").read()
    open(good, "wb").write(raw[:-8])                 # truncated data
    with pytest.raises(cruna.CrunaError) as e:
        cruna.read_snapshot(good)
    assert e.value.code == -7


def test_file_system_failures_are_io_errors(tmp_path):
    missing = str(tmp_path / "no_such_dir")
    with pytest.raises(cruna.CrunaError) as e:
        cruna.write_snapshot(missing + "/snap.bin", np.ones((2, 2, 2, 5), order="F"))
    assert e.value.code == -7                        # the .tmp file cannot be opened
    with pytest.raises(cruna.CrunaError) as e:
        cruna.read_snapshot(str(tmp_path / "absent.bin"))
    assert e.value.code == -7
    with pytest.raises(cruna.CrunaError) as e:
        cruna.write_restart(missing, 1, 2)
    assert e.value.code == -7
    with pytest.raises(cruna.CrunaError) as e:
        cruna.io_fname(str(tmp_path), "no_such_type")
    assert e.value.code == -1                        # an argument error, not I/O


def test_restartfile_round_trip_and_absence(tmp_path):
    w = str(tmp_path)
    assert cruna.read_restart(w) is None             # cruna_hpc.f90:127-131: not found, start from 0
    cruna.write_restart(w, 2, 345)
    assert cruna.read_restart(w) == (2, 345)
    cruna.write_restart(w, 3, 7)                     # overwritten, as with file_overwrite_optin
    assert cruna.read_restart(w) == (3, 7)


@pytest.mark.parametrize("ns,nt,steps", [(1, 0, 10), (1, 5, 10), (1, 9, 10), (1, 10, 10), (2, 3, 10),
                                         (4, 1, 7), (1, 0, 1), (3, 1, 1)])
def test_restart_start_arithmetic(ns, nt, steps):
    # cruna_hpc.f90:143-145, restated
    total = (ns - 1) * steps + nt + 1
    s0 = total // steps + 1
    assert cruna.restart_start(ns, nt, steps) == (s0, total - (s0 - 1) * steps)
