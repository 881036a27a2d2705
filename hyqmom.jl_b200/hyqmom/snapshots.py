"""Snapshot stream with the reference's key layout (src/simulation_runner.jl:282-330, 669-698, 733-743):

    meta/params, meta/snapshot_interval, meta/n_snapshots, grid/<field>,
    snapshots/%06d/{M, t, step, S, C}

The reference streams these keys into a JLD2 (HDF5) file.  No HDF5 writer is
available to this package, so the same keys are streamed into a NumPy
``.npz`` archive instead, and the file is named for that format (a requested
``*.jld2`` name becomes ``*.npz``).  Each snapshot is written to the archive
inside ``write()`` and its arrays are released at once, as the reference does
(src/simulation_runner.jl:669-698), so host memory stays at one snapshot and a
crash keeps every snapshot written before it.  ``np.load(filename)`` reads the
archive; member ``snapshots/000001/M`` is the initial condition.

The reference always writes S and C (``save_standardized = save_central =
true``, src/simulation_runner.jl:109-110); ``write()`` takes them as optional
so a caller may leave either out.
"""
import os
import zipfile

import numpy as np


def npz_name(filename):
    """The archive's file name: a ``.jld2`` suffix is replaced by ``.npz``."""
    root, ext = os.path.splitext(filename)
    if ext == ".jld2":
        return root + ".npz"
    return filename if ext == ".npz" else filename + ".npz"


class SnapshotWriter:
    def __init__(self, filename, params, interval):
        self.filename = npz_name(filename)
        self.count = 0
        self._zip = zipfile.ZipFile(self.filename, "w", compression=zipfile.ZIP_STORED, allowZip64=True)
        self._put("meta/snapshot_interval", np.int64(interval))
        self._put("meta/params", np.array(repr({k: v for k, v in params.items() if not k.startswith("ic_")})))

    def _put(self, key, arr):
        with self._zip.open(key + ".npy", "w", force_zip64=True) as f:
            np.lib.format.write_array(f, np.asanyarray(arr), allow_pickle=False)
        self._zip.fp.flush()

    def write(self, M, t, step, S=None, C=None):
        """Append snapshot number count+1 and flush it to the file."""
        self.count += 1
        key = "snapshots/%06d/" % self.count
        self._put(key + "M", M)
        self._put(key + "t", np.float64(t))
        self._put(key + "step", np.int64(step))
        if S is not None:
            self._put(key + "S", S)
        if C is not None:
            self._put(key + "C", C)

    def close(self, grid):
        if self._zip is None:
            return
        self._put("meta/n_snapshots", np.int64(self.count))
        for k, v in grid.items():
            self._put("grid/" + k, np.asarray(v))
        self._zip.close()
        self._zip = None

    def __del__(self):
        try:
            if self._zip is not None:
                self._zip.close()
        except Exception:
            pass
