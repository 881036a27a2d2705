"""Snapshot stream with the reference's key layout (src/simulation_runner.jl:282-330, 669-698, 733-743):

    meta/params, meta/snapshot_interval, meta/n_snapshots, grid,
    snapshots/%06d/{M, t, step, S, C}

Written as a NumPy ``.npz`` archive whose member names are those keys (the
reference writes the same keys into a JLD2 file).
"""
import numpy as np


class SnapshotWriter:
    def __init__(self, filename, params, interval):
        self.filename = filename
        self.count = 0
        self._items = {"meta/snapshot_interval": np.int64(interval),
                       "meta/params": np.array(repr({k: v for k, v in params.items() if not k.startswith("ic_")}))}

    def write(self, M, t, step, S=None, C=None):
        self.count += 1
        key = "snapshots/%06d/" % self.count
        self._items[key + "M"] = np.asarray(M)
        self._items[key + "t"] = np.float64(t)
        self._items[key + "step"] = np.int64(step)
        if S is not None:
            self._items[key + "S"] = np.asarray(S)
        if C is not None:
            self._items[key + "C"] = np.asarray(C)

    def close(self, grid):
        self._items["meta/n_snapshots"] = np.int64(self.count)
        for k, v in grid.items():
            self._items["grid/" + k] = np.asarray(v)
        with open(self.filename, "wb") as f:
            np.savez(f, **self._items)
