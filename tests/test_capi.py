"""The C-ABI library loads here (no GPU) and exports every symbol include/*.h declares;
host-side argument checks return MR_ERR_INVALID before any launch."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import build as B


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(B.LIBPATH):
        B.build()
    return N.load()


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:int|int64_t|void|const\s+char\s*\*)\s*(mr_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 8
    for name in names:
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, f"{name} has no binding"


def test_struct_sizes_and_version(lib):
    assert lib.mr_abi_version() == 1
    assert [lib.mr_struct_size(i) for i in range(5)] == [40, 64, 256, 16, 32]
    assert lib.mr_struct_size(9) == -1
    assert lib.mr_status_string(0) == b"ok"
    assert lib.mr_status_string(-1) == b"invalid argument"


def test_invalid_arguments_are_rejected_on_the_host(lib):
    assert lib.mr_backproject(None, None, None, None, 0, None, None) == N.MR_ERR_INVALID
    ring = N.MrRing()
    ring.data = 0
    assert lib.mr_backproject(ctypes.byref(ring), None, None, None, 1, None, None) == N.MR_ERR_INVALID
    ring.data = 1 << 20          # never dereferenced: the checks below fail first
    ring.rows, ring.cols, ring.col_pitch, ring.slot_stride = 4, 8, 4, 32
    ring.dtype, ring.kind = N.MR_F32, N.MR_CONE
    fake = ctypes.c_void_p(1 << 20)
    assert lib.mr_backproject(ctypes.byref(ring), fake, fake, fake, 1, fake, None) == N.MR_ERR_INVALID
    ring.col_pitch = 8
    ring.kind = 7
    assert lib.mr_backproject(ctypes.byref(ring), fake, fake, fake, 1, fake, None) == N.MR_ERR_INVALID
    ring.kind = N.MR_CONE
    # FFT length shorter than 2 * cols is refused
    assert lib.mr_filter_f32(fake, 8, 8, 1, fake, fake, fake, 3, ctypes.byref(ring), None) == N.MR_ERR_INVALID
    assert lib.mr_ingest_u16(fake, 8, 8, 0, 0, fake, fake, 1, fake, fake, fake, 5,
                             ctypes.byref(ring), None) == N.MR_ERR_INVALID
    assert lib.mr_rotate_f32(fake, fake, 4, 1, 8, 1.0, None) == N.MR_ERR_INVALID
    assert lib.mr_gaussian_axis_f32(fake, fake, 4, 1, 8, 1, 2, fake, 3, None) == N.MR_ERR_INVALID


def test_plan_tiles_argument_checks(lib):
    n = ctypes.c_int64()
    assert lib.mr_plan_tiles(None, 1, None, 0, ctypes.byref(n)) == N.MR_ERR_INVALID
    g = np.zeros(1, N.GRID_DTYPE)
    g["n_i"] = -1
    assert lib.mr_plan_tiles(g.ctypes.data, 1, None, 0, ctypes.byref(n)) == N.MR_ERR_INVALID
