"""Host-side checks that need no GPU: the C-ABI library loads and exports
every entry point that include/*.h declares."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(cls_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cls_create" in names and "cls_backward" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    import cls_b200
    lib = ctypes.CDLL(cls_b200._capi.lib_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_gpu_reports_error_not_crash():
    """Without a GPU, creation must fail with an error code and a message."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import cls_b200
    import numpy as np
    r = cls_b200.Robot(np.zeros((2, 3)), np.array([[0, 1, 0.1, 1e4, 0.0]]), hidden=[4])
    with pytest.raises(cls_b200._capi.ClsError):
        cls_b200.MassSpringBatch([r], [0])


def test_invalid_arguments_rejected_before_any_device_work():
    import cls_b200
    import numpy as np
    bad = cls_b200.Robot(np.zeros((2, 3)), np.array([[0, 5, 0.1, 1e4, 0.0]]), hidden=[4])
    with pytest.raises(cls_b200._capi.ClsError, match="endpoint"):
        cls_b200.MassSpringBatch([bad], [0])


def test_shape_and_table_entry_points_reject_null_handles():
    """Launch-shape, autotuner, spring-table and phase-clock calls return
    CLS_ERR_INVALID for a NULL handle or output pointer (no device work)."""
    import ctypes
    import cls_b200
    lib = cls_b200._capi.load()
    inv = -1  # CLS_ERR_INVALID
    i32 = ctypes.c_int32()
    table = (cls_b200._capi.LaunchShape * 4)()
    clocks = (ctypes.c_uint64 * 32)()
    assert lib.cls_set_launch_shape(None, 256, 1, -1) == inv
    assert lib.cls_get_launch_shape(None, ctypes.byref(i32), ctypes.byref(i32), None) == inv
    assert lib.cls_autotune(None, 0, 1, table, 4, ctypes.byref(i32)) == inv
    assert lib.cls_autotune(None, 0, 1, None, 4, ctypes.byref(i32)) == inv   # table missing
    assert lib.cls_set_spring_tables(None, 0) == inv
    assert lib.cls_spring_tables(None, ctypes.byref(i32)) == inv
    assert lib.cls_phase_read(None, clocks) == inv
