"""Host logic of the launch-shape autotuner (hyqmom.autotune): the JSON cache
keyed by device and workload, and the workload keys; no GPU needed."""
import json

from hyqmom import autotune, ic


def test_cache_round_trip_and_keys(tmp_path, monkeypatch):
    path = str(tmp_path / "sub" / "tune.json")
    monkeypatch.setenv(autotune.CACHE_ENV, path)
    assert autotune.cache_path() == path
    assert autotune.load_cache() == {}  # a missing file reads as empty
    autotune._store("devA", "k1", {"hll": 6}, None)
    autotune._store("devA", "k2", {"hll": 2}, None)
    autotune._store("devB", "k1", {"hll": 0}, None)
    assert autotune._lookup("devA", "k1", None) == {"hll": 6}
    assert autotune._lookup("devB", "k1", None) == {"hll": 0}
    assert autotune._lookup("devB", "k2", None) is None
    with open(path) as f:
        assert json.load(f) == {"devA": {"k1": {"hll": 6}, "k2": {"hll": 2}}, "devB": {"k1": {"hll": 0}}}
    with open(path, "w") as f:
        f.write("{not json")
    assert autotune.load_cache() == {}  # a damaged cache is ignored, not fatal


def test_workload_keys():
    a = ic.default_params(Nx=24, Ny=20, Nz=16)
    b = ic.default_params(Nx=16, Ny=16, Nz=12)
    assert autotune.solver_key(a, "plain") == "solver|24x20x16|plain"
    assert autotune.solver_key(a, "plain") != autotune.solver_key(a, "learned")
    k1, k2 = autotune.batch_key([a, b], "plain"), autotune.batch_key([b, a], "plain")
    assert k1.startswith("batch|2|plain|") and k1 != k2  # member order is part of the workload
    assert autotune.batch_key([a, b], "plain") == k1
