"""TEST INFRASTRUCTURE ONLY. ctypes front of oracle/bp_oracle.c (the C restatement of
minirecast recon.py:156-219 bp_cone_numba / bp_parallel_numba / _bil_nb)."""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "liboracle_bp.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.c_long


def build():
    """Compile the C oracle with gcc (oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIBPATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIBPATH) or (
                os.path.getmtime(_LIBPATH) < os.path.getmtime(os.path.join(_HERE, "bp_oracle.c"))):
            build()
        L = ctypes.CDLL(_LIBPATH)
        for name in ("oracle_bp_cone_f32", "oracle_bp_cone_f64"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _L, _L, _L, _D, _D, _D, _D, _D, _D, _D,
                                         _D, _L, ctypes.c_double, _D]
            getattr(L, name).restype = None
        for name in ("oracle_bp_parallel_f32", "oracle_bp_parallel_f64"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _L, _L, _L, _D, _D, ctypes.c_double,
                                         ctypes.c_double, _D, _L, ctypes.c_double, ctypes.c_double, _D]
            getattr(L, name).restype = None
        L.oracle_threads.argtypes = [ctypes.c_int]
        L.oracle_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def threads(n=0):
    return lib().oracle_threads(int(n))


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_D)


def bp_cone(q, S, D, UU, VV, Nn, SDD, SOD, pts, scale):
    """bp_cone_numba (recon.py:193-219): q [A,R,C] f32 or f64, f64 accumulation."""
    q = np.ascontiguousarray(q)
    fn = lib().oracle_bp_cone_f64 if q.dtype == np.float64 else lib().oracle_bp_cone_f32
    q = q if q.dtype == np.float64 else np.ascontiguousarray(q, dtype=np.float32)
    A, R, C = q.shape
    keep = [_d(x) for x in (S, D, UU, VV, Nn, SDD, SOD, pts)]
    pts_a = keep[-1][0]
    M = pts_a.size // 3
    out = np.zeros(M)
    fn(q.ctypes.data, A, R, C, *[k[1] for k in keep], M, float(scale), out.ctypes.data_as(_D))
    return out


def bp_parallel(q, cos_t, sin_t, pu, pv, pts, scale, col_shift):
    """bp_parallel_numba (recon.py:175-191)."""
    q = np.ascontiguousarray(q)
    fn = lib().oracle_bp_parallel_f64 if q.dtype == np.float64 else lib().oracle_bp_parallel_f32
    q = q if q.dtype == np.float64 else np.ascontiguousarray(q, dtype=np.float32)
    A, R, C = q.shape
    c, s, p = _d(cos_t), _d(sin_t), _d(pts)
    M = p[0].size // 3
    out = np.zeros(M)
    fn(q.ctypes.data, A, R, C, c[1], s[1], float(pu), float(pv), p[1], M, float(scale),
       float(col_shift), out.ctypes.data_as(_D))
    return out
