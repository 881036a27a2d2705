"""Host logic of the snapshot stream (hyqmom.snapshots): the reference's key
layout (src/simulation_runner.jl:282-330, 669-698), each snapshot written to
the file as it comes; no GPU needed."""
import zipfile

import numpy as np

from hyqmom import snapshots


def test_names():
    assert snapshots.npz_name("run.jld2") == "run.npz"
    assert snapshots.npz_name("run.npz") == "run.npz"
    assert snapshots.npz_name("run") == "run.npz"


def test_key_layout_and_values(tmp_path):
    w = snapshots.SnapshotWriter(str(tmp_path / "out.jld2"), {"Nx": 4, "Ma": 1.0, "ic_jets": [object()]}, 2)
    rng = np.random.default_rng(0)
    Ms = [rng.standard_normal((4, 3, 2, 35)) for _ in range(3)]
    for k, M in enumerate(Ms):
        w.write(M, 0.1 * k, 2 * k + 1, S=M + 1.0, C=M - 1.0 if k != 1 else None)
    w.close({"xm": np.arange(4.0), "dx": 0.25})
    z = np.load(str(tmp_path / "out.npz"))
    assert int(z["meta/snapshot_interval"]) == 2 and int(z["meta/n_snapshots"]) == 3
    assert "ic_jets" not in str(z["meta/params"]) and "'Nx': 4" in str(z["meta/params"])
    for k, M in enumerate(Ms):
        key = "snapshots/%06d/" % (k + 1)
        assert np.array_equal(z[key + "M"], M) and float(z[key + "t"]) == 0.1 * k and int(z[key + "step"]) == 2 * k + 1
        assert np.array_equal(z[key + "S"], M + 1.0)
        assert (key + "C" in z.files) == (k != 1)
    assert np.array_equal(z["grid/xm"], np.arange(4.0)) and float(z["grid/dx"]) == 0.25


def test_snapshots_reach_the_file_as_they_are_written(tmp_path):
    """Each write reaches the file at once: before close() (as after a
    crash) every member written so far is on disk with its local header, from
    which a zip tool can rebuild the archive."""
    path = str(tmp_path / "crash.npz")
    w = snapshots.SnapshotWriter(path, {"Nx": 2}, 1)
    M = np.ones((2, 2, 1, 35))
    w.write(M, 0.0, 1)
    w.write(2 * M, 0.5, 2)
    with open(path, "rb") as f:
        data = f.read()
    assert data.count(b"PK\x03\x04") == 2 + 6  # meta/snapshot_interval, meta/params, 2 x (M, t, step)
    assert data.count(b"PK\x01\x02") == 0  # no central directory until close()
    w.close({})
    assert zipfile.is_zipfile(path)
