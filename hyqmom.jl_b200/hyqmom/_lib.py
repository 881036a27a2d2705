"""ctypes binding of libhyqmom_b200.so (declared in include/hyqmom.h).

The library is the only compute path: if it is missing or fails to load the
import raises; there is no CPU fallback.
"""
import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_NAME = "libhyqmom_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

HYQ_OK = 0
ERRORS = {-1: "HYQ_EINVAL", -2: "HYQ_ECUDA", -3: "HYQ_ENONFINITE", -4: "HYQ_ETIMEOUT", -5: "HYQ_ENOMEM"}


class HyqParams(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32), ("flag2D", ctypes.c_int32),
                ("positivity", ctypes.c_int32), ("device", ctypes.c_int32), ("nnmax", ctypes.c_int64),
                ("tmax", ctypes.c_double), ("Kn", ctypes.c_double), ("Ma", ctypes.c_double), ("CFL", ctypes.c_double),
                ("dtmax", ctypes.c_double), ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymin", ctypes.c_double), ("ymax", ctypes.c_double), ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
                ("mode", ctypes.c_int32), ("symmetry_check_interval", ctypes.c_int32)]


class HyqIcRegion(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("everywhere", ctypes.c_int32), ("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3),
                ("i0", ctypes.c_int32), ("i1", ctypes.c_int32), ("j0", ctypes.c_int32), ("j1", ctypes.c_int32),
                ("k0", ctypes.c_int32), ("k1", ctypes.c_int32)]


# hyq_params.mode
MODE_PLAIN, MODE_LEARNED, MODE_CERTIFIED = 0, 1, 2
MODES = {"plain": MODE_PLAIN, "learned": MODE_LEARNED, "certified": MODE_CERTIFIED}
NET_PARAMS = 38406  # HYQ_NET_PARAMS
# launch variants (hyq_set_variant) and batch schedules (hyq_batch_set_schedule)
KERNEL_HLL, KERNEL_CORR = 0, 1
BATCH_BRANCHES, BATCH_FUSED = 0, 1


class HyqStats(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("dt", ctypes.c_double), ("vmax", ctypes.c_double), ("nn", ctypes.c_int64),
                ("done", ctypes.c_int32), ("status", ctypes.c_int32), ("stage_cells", ctypes.c_int64),
                ("fallback_cells", ctypes.c_int64), ("dense_mask", ctypes.c_int32), ("worst_dir", ctypes.c_int32),
                ("vmax_first", ctypes.c_double * 3), ("worst_cell", ctypes.c_int64), ("maxdiff", ctypes.c_double),
                ("maxdiff_step", ctypes.c_int64)]


class HyqError(RuntimeError):
    pass


_lib = None

# exported symbols (include/hyqmom.h)
SYMBOLS = ["hyq_abi_version", "hyq_create", "hyq_destroy", "hyq_last_error", "hyq_set_state", "hyq_get_state",
           "hyq_set_state_device", "hyq_get_state_device", "hyq_set_clock", "hyq_advance", "hyq_advance_async",
           "hyq_synchronize", "hyq_stats_get", "hyq_advance_timed", "hyq_step_host", "hyq_get_SC", "hyq_stream", "hyq_cells_flux_closure",
           "hyq_cells_eigenvalues", "hyq_cells_closure_eigs", "hyq_cells_collision", "hyq_cells_phase_A", "hyq_step_noalloc", "hyq_batch_create", "hyq_batch_destroy", "hyq_batch_size",
           "hyq_batch_member", "hyq_batch_stream", "hyq_batch_advance_async", "hyq_batch_advance", "hyq_reset_counters",
           "hyq_set_wavespeed_net", "hyq_net_image_bytes", "hyq_net_tile_bytes", "hyq_net_scratch_bytes", "hyq_net_pack",
           "hyq_net_features", "hyq_net_forward", "hyq_net_train_batch", "hyq_net_adam", "hyq_cells_wavespeed_targets", "hyq_set_state_ic", "hyq_step_begin", "hyq_step_end", "hyq_copy_layers", "hyq_set_spacing",
           "hyq_variant_count", "hyq_set_variant", "hyq_batch_set_variant", "hyq_batch_set_schedule", "hyq_batch_schedule"]
NOALLOC_MAX_CELLS = 16384  # HYQ_NOALLOC_MAX_CELLS


def load(path=None):
    """Load the library (raises if the CUDA build is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise HyqError(f"{LIB_NAME} not built (expected at {path}); run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    vp, dp, i64, i32, dbl = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64, ctypes.c_int32, ctypes.c_double
    lib.hyq_abi_version.restype = ctypes.c_int
    lib.hyq_create.argtypes = [ctypes.POINTER(HyqParams), ctypes.POINTER(vp)]
    lib.hyq_destroy.argtypes = [vp]
    lib.hyq_destroy.restype = None
    lib.hyq_last_error.argtypes = [vp]
    lib.hyq_last_error.restype = ctypes.c_char_p
    for nm in ("hyq_set_state", "hyq_get_state", "hyq_set_state_device", "hyq_get_state_device"):
        getattr(lib, nm).argtypes = [vp, vp]
    lib.hyq_set_clock.argtypes = [vp, dbl, i64]
    lib.hyq_advance.argtypes = [vp, i64, dp, ctypes.POINTER(i64), ctypes.POINTER(i32)]
    lib.hyq_advance_async.argtypes = [vp, i64]
    lib.hyq_synchronize.argtypes = [vp]
    lib.hyq_advance_timed.argtypes = [vp, i64, ctypes.POINTER(ctypes.c_float)]
    lib.hyq_step_host.argtypes = [vp, vp, vp, i32, dp, ctypes.POINTER(i64), ctypes.POINTER(i32)]
    lib.hyq_stats_get.argtypes = [vp, ctypes.POINTER(HyqStats)]
    lib.hyq_get_SC.argtypes = [vp, vp, vp]
    lib.hyq_stream.argtypes = [vp]
    lib.hyq_stream.restype = vp
    lib.hyq_cells_flux_closure.argtypes = [vp, i64, i32, dbl, vp, vp, vp, vp, vp]
    lib.hyq_cells_eigenvalues.argtypes = [vp, i64, i32, i32, dbl, i32, vp, vp, vp]
    lib.hyq_cells_closure_eigs.argtypes = [vp, i64, vp, vp]
    lib.hyq_cells_collision.argtypes = [vp, i64, dbl, dbl, i32, vp, vp]
    lib.hyq_cells_phase_A.argtypes = [vp, i64, i32, dbl, i32, vp, vp, vp, vp, vp, vp]
    lib.hyq_step_noalloc.argtypes = [ctypes.POINTER(HyqParams), vp, ctypes.POINTER(HyqStats), vp]
    lib.hyq_batch_create.argtypes = [ctypes.POINTER(HyqParams), i32, ctypes.POINTER(vp)]
    lib.hyq_batch_destroy.argtypes = [vp]
    lib.hyq_batch_destroy.restype = None
    lib.hyq_batch_size.argtypes = [vp]
    lib.hyq_batch_size.restype = i32
    lib.hyq_batch_member.argtypes = [vp, i32]
    lib.hyq_batch_member.restype = vp
    lib.hyq_batch_stream.argtypes = [vp]
    lib.hyq_batch_stream.restype = vp
    lib.hyq_batch_advance_async.argtypes = [vp, i64]
    lib.hyq_batch_advance.argtypes = [vp, i64, ctypes.POINTER(i32), ctypes.POINTER(i32)]
    flt = ctypes.c_float
    lib.hyq_reset_counters.argtypes = [vp]
    lib.hyq_set_wavespeed_net.argtypes = [vp, vp, dbl]
    for nm in ("hyq_net_image_bytes", "hyq_net_tile_bytes"):
        getattr(lib, nm).restype = i64
    lib.hyq_net_scratch_bytes.argtypes = [i32]
    lib.hyq_net_scratch_bytes.restype = i64
    lib.hyq_net_pack.argtypes = [vp, vp, vp]
    lib.hyq_net_features.argtypes = [vp, i64, vp, vp]
    lib.hyq_net_forward.argtypes = [vp, vp, i64, vp, vp, vp]
    lib.hyq_net_train_batch.argtypes = [vp, vp, vp, i64, vp, i32, flt, vp, vp, i32, vp, vp, vp]
    lib.hyq_net_adam.argtypes = [vp, vp, vp, vp, i32, flt, flt, flt, flt, flt, i32, vp, vp]
    lib.hyq_cells_wavespeed_targets.argtypes = [vp, i64, i32, dbl, i32, vp, vp, vp]
    lib.hyq_set_state_ic.argtypes = [vp, vp, vp, vp, dbl, dbl, dbl, vp, i32, vp, vp]
    lib.hyq_step_begin.argtypes = [vp, vp]
    lib.hyq_step_end.argtypes = [vp, vp]
    lib.hyq_copy_layers.argtypes = [vp, i32, i32, vp, i32]
    lib.hyq_set_spacing.argtypes = [vp, dbl, dbl, dbl]
    lib.hyq_variant_count.argtypes = [i32]
    lib.hyq_variant_count.restype = i32
    lib.hyq_set_variant.argtypes = [vp, i32, i32]
    lib.hyq_batch_set_variant.argtypes = [vp, i32, i32]
    lib.hyq_batch_set_schedule.argtypes = [vp, i32]
    lib.hyq_batch_schedule.argtypes = [vp]
    lib.hyq_batch_schedule.restype = i32
    _lib = lib
    return lib


def check(rc, ctx=None):
    if rc != HYQ_OK:
        msg = load().hyq_last_error(ctx).decode() if load() else ""
        raise HyqError(f"{ERRORS.get(rc, rc)}: {msg}")
