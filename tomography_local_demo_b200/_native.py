"""ctypes binding of the sm_100a library (include/minirecast_b200.h).

The library is the only compute path: there is no CPU fallback. If it is missing,
every call raises RuntimeError naming the build step.
"""
import collections
import ctypes
import os
import threading

import numpy as np

from . import build as _build

MR_OK = 0
MR_ERR_INVALID = -1
MR_ERR_CUDA = -2
MR_ERR_UNSUPPORTED = -3
MR_ERR_TIMEOUT = -4
MR_ERR_SCRATCH_LIMIT = -5
MR_ERR_CAPTURE = -6
MR_NOALLOC_MAX_TILES = 1 << 31

MR_F32, MR_BF16, MR_F16, MR_U16 = 0, 1, 2, 3
MR_CORRECT_FLEXRAY, MR_CORRECT_HDF5 = 0, 1
MR_PARALLEL, MR_CONE = 0, 1
MR_GRID_MASK_BOX, MR_GRID_POINTS = 1, 2

# numpy mirrors of the ABI structs (checked against mr_struct_size at load time)
VIEW_DTYPE = np.dtype([("pu", "<f4", 4), ("pv", "<f4", 4), ("pw", "<f4", 4), ("uv", "<f4"),
                       ("qscale", "<f4"), ("pad", "<f4", 2)], align=True)
GRID_DTYPE = np.dtype([("origin", "<f4", 3), ("step_i", "<f4", 3), ("step_j", "<f4", 3),
                       ("step_k", "<f4", 3), ("cor_shift", "<f4"), ("scale", "<f4"),
                       ("n_i", "<i4"), ("n_j", "<i4"), ("n_k", "<i4"), ("n_views", "<i4"),
                       ("flags", "<i4"), ("tilt", "<f4"), ("out_offset", "<i8"),
                       ("out_stride_i", "<i8"), ("out_stride_j", "<i8"), ("out_stride_k", "<i8"),
                       ("points", "<u8"), ("tilt_cos", "<f4"), ("tilt_sin", "<f4"), ("mask_c", "<f8", 3),
                       ("mask_ej", "<f8", 3), ("mask_ei", "<f8", 3), ("mask_half", "<f8"),
                       ("mask_delta", "<f8"), ("box", "<f8", 3), ("view_begin", "<i4"), ("accumulate", "<i4"),
                       ("pad2", "<i8")], align=True)
TILE_DTYPE = np.dtype([("grid", "<i4"), ("i0", "<i4"), ("j0", "<i4"), ("k", "<i4")], align=True)
FILTER_VIEW_DTYPE = np.dtype([("a0", "<f4"), ("da", "<f4"), ("b0", "<f4"), ("db", "<f4"),
                              ("sdd", "<f4"), ("gain", "<f4"), ("out_scale", "<f4"),
                              ("slot", "<i4")], align=True)


class MrRing(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("dtype", ctypes.c_int32), ("kind", ctypes.c_int32),
                ("rows", ctypes.c_int32), ("cols", ctypes.c_int32), ("col_pitch", ctypes.c_int32),
                ("n_slots", ctypes.c_int32), ("slot_stride", ctypes.c_int64)]


# every exported symbol of include/minirecast_b200.h with (restype, argtypes)
_P = ctypes.c_void_p
_I32, _I64 = ctypes.c_int32, ctypes.c_int64
SIGNATURES = {
    "mr_abi_version": (ctypes.c_int, []),
    "mr_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "mr_last_cuda_error": (ctypes.c_char_p, []),
    "mr_struct_size": (ctypes.c_int, [ctypes.c_int]),
    "mr_bp_tile_shape": (None, [ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "mr_plan_tiles": (ctypes.c_int, [_P, _I32, _P, _I64, ctypes.POINTER(_I64)]),
    "mr_backproject": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _I64, _P, _P]),
    "mr_backproject_staged": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _I64, _P, _P, _P]),
    "mr_backproject_persistent": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _P, _I64, _P, _P, _P, _P]),
    "mr_backproject_persistent_noalloc": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _P, _I64, _P, _P, _P]),
    "mr_backproject_matched": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _I64, _P, _P]),
    "mr_project_adjoint": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _I64, _P, _P]),
    "mr_bp_grad_geom": (ctypes.c_int, [ctypes.POINTER(MrRing), _P, _P, _P, _I64, _P, _P, _P]),
    "mr_filter_f32": (ctypes.c_int, [_P, _I64, _I64, _I32, _P, _P, _P, _I32,
                                     ctypes.POINTER(MrRing), _P]),
    "mr_ingest_u16": (ctypes.c_int, [_P, _I64, _I64, _I32, _I32, _P, _P, _I32, _P, _P, _P, _I32,
                                     ctypes.POINTER(MrRing), _P]),
    "mr_toeplitz_image_bytes": (ctypes.c_int64, [_I32]),
    "mr_toeplitz_image": (ctypes.c_int, [_P, _I32, _I32, _I32, _P, ctypes.POINTER(ctypes.c_float)]),
    "mr_filter_f32_tc": (ctypes.c_int, [_P, _I64, _I64, _I32, _P, _P, _I32, ctypes.c_float, ctypes.c_float, _I32,
                                        ctypes.POINTER(MrRing), _P, _P]),
    "mr_ingest_u16_tc": (ctypes.c_int, [_P, _I64, _I64, _I32, _I32, _P, _P, _I32, _P, _P, _I32, ctypes.c_float,
                                        _I32, ctypes.POINTER(MrRing), _P, _P]),
    "mr_slice_entropy": (ctypes.c_int, [_P, _I32, _I64, _I32, _I32, _P, _P]),
    "mr_correct_u16": (ctypes.c_int, [_P, _I64, _I64, _I32, _I32, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P,
                                       _I64, _I32, _P, _I64, _I64, _P]),
    "mr_mc_blocks": (_I64, [_I32, _I32, _I32]),
    "mr_mc_table": (ctypes.c_int, [_P]),
    "mr_mc_count": (ctypes.c_int, [_P, _I32, _I32, _I32, ctypes.c_float, _P, _P]),
    "mr_mc_emit": (ctypes.c_int, [_P, _I32, _I32, _I32, ctypes.c_float, _P, ctypes.c_double, _P, _I64, _P, _P,
                                  _P]),
    "mr_volume_workspace_bytes": (_I64, []),
    "mr_volume_stats": (ctypes.c_int, [_P, _I64, _P, _P, _P]),
    "mr_volume_select": (ctypes.c_int, [_P, _I64, _P, _I32, ctypes.c_uint32, ctypes.c_uint32, _P, _P, _P]),
    "mr_volume_histogram": (ctypes.c_int, [_P, _I64, _P, _I32, ctypes.c_double, ctypes.c_double, _P, _P]),
    "mr_rotate_f32": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, ctypes.c_double, _P]),
    "mr_gaussian_axis_f32": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _I32, _I32, _P, _I32, _P]),
}

_lock = threading.Lock()
_lib = None


def library_path():
    return _build.LIBPATH


def load():
    """Load (once) and return the ctypes library; raise if it was never built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA library {path} is missing: run "
                               "`python -m tomography_local_demo_b200.build` (or __graft_entry__.build())")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        sizes = {0: ctypes.sizeof(MrRing), 1: VIEW_DTYPE.itemsize, 2: GRID_DTYPE.itemsize,
                 3: TILE_DTYPE.itemsize, 4: FILTER_VIEW_DTYPE.itemsize}
        for which, size in sizes.items():
            got = lib.mr_struct_size(which)
            if got != size:
                raise RuntimeError(f"ABI struct {which} size mismatch: library {got}, binding {size}")
        _lib = lib
        return lib


def check(status, what):
    """Map a status code to the exception the reference raises for the same condition."""
    if status == MR_OK:
        return
    msg = f"{what}: {load().mr_status_string(status).decode()} (status {status})"
    if status == MR_ERR_CUDA:
        msg += f": {load().mr_last_cuda_error().decode()}"
    if status == MR_ERR_INVALID:
        raise ValueError(msg)
    if status == MR_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


def tile_shape():
    ti, tj = _I32(), _I32()
    load().mr_bp_tile_shape(ctypes.byref(ti), ctypes.byref(tj))
    return ti.value, tj.value


_TILE_SHAPE = None


_PLAN_CACHE = collections.OrderedDict()     # (grid bytes, band axis) -> read-only tile array
_PLAN_CACHE_MAX = 64
_PLAN_LOCK = threading.Lock()


def plan_tiles(grids, band_axis=None):
    """plan_tiles_uncached, memoised on the grid records' bytes and the band axis: a
    repeated request list (a viewer re-slicing, a server replaying, a bench step) reuses
    its tile list instead of re-planning it on the host. The returned array is read-only."""
    grids = np.ascontiguousarray(grids, dtype=GRID_DTYPE)
    key = (grids.tobytes(), None if band_axis is None else tuple(float(x) for x in band_axis))
    with _PLAN_LOCK:
        hit = _PLAN_CACHE.get(key)
        if hit is not None:
            _PLAN_CACHE.move_to_end(key)
            return hit
    tiles = plan_tiles_uncached(grids, band_axis)
    tiles.flags.writeable = False
    with _PLAN_LOCK:
        _PLAN_CACHE[key] = tiles
        if len(_PLAN_CACHE) > _PLAN_CACHE_MAX:
            _PLAN_CACHE.popitem(last=False)
    return tiles


def plan_tiles_uncached(grids, band_axis=None):
    """Tiles (numpy TILE_DTYPE array) covering the grids (numpy GRID_DTYPE array).

    band_axis: the orbit's rotation axis (the detector's row direction). When given, the
    tiles of regular grids are ordered by their centre's position along it, highest first,
    across all grids of the launch. Every view projects tiles at one height onto the same
    band of detector rows, so the tiles in flight together read one band of the filtered
    ring instead of footprints spread over the whole detector: their footprint loads then
    mostly hit L2 (the ring of a scan is larger than L2). The result is the same bit for
    bit in any order (each tile is summed by one cluster); on a 600-view scan the staged
    back-projection of three oblique slices ran 3.6 % faster (highest first measured 1-2 %
    faster than lowest first)."""
    global _TILE_SHAPE
    grids = np.ascontiguousarray(grids, dtype=GRID_DTYPE)
    lib = load()
    n = _I64()
    check(lib.mr_plan_tiles(grids.ctypes.data, len(grids), None, 0, ctypes.byref(n)), "plan_tiles")
    tiles = np.empty(n.value, dtype=TILE_DTYPE)
    check(lib.mr_plan_tiles(grids.ctypes.data, len(grids), tiles.ctypes.data, len(tiles),
                            ctypes.byref(n)), "plan_tiles")
    if band_axis is not None and len(tiles) > 1 and not (grids["flags"] & MR_GRID_POINTS).any():
        if _TILE_SHAPE is None:
            _TILE_SHAPE = tile_shape()
        a = np.asarray(band_axis, dtype=np.float64)
        gi = tiles["grid"]
        o = grids["origin"].astype(np.float64) @ a
        si = grids["step_i"].astype(np.float64) @ a
        sj = grids["step_j"].astype(np.float64) @ a
        sk = grids["step_k"].astype(np.float64) @ a
        key = (o[gi] + (tiles["i0"] + 0.5 * (_TILE_SHAPE[0] - 1)) * si[gi]
               + (tiles["j0"] + 0.5 * (_TILE_SHAPE[1] - 1)) * sj[gi] + tiles["k"] * sk[gi])
        tiles = tiles[np.argsort(-key, kind="stable")]
    return tiles
