"""The SHOCK-side binding (shock_b200/dropin/GPU.c) as built into the
drop-in harness: it loads without a GPU and exports the entry points that
shock_b200/dropin/GPU.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libshockdropin_w5_3d.so")


def test_dropin_binding_exports():
    if not os.path.exists(LIB):
        pytest.skip("drop-in harness not built (make -C oracle with the reference sources)")
    header = open(os.path.join(ROOT, "shock_b200", "dropin", "GPU.h")).read()
    names = re.findall(r"\b(GPU_\w+)\s*\(", header)
    assert set(names) == {"GPU_Create", "GPU_CalcRungeKutta", "GPU_CheckNAN", "GPU_SyncHost", "GPU_UploadState",
                          "GPU_Destroy", "GPU_EnableHistories", "GPU_WriteValuesForPressureHistory",
                          "GPU_WriteValuesForVelocityHistory", "GPU_EnableFilm", "GPU_SampleFilm", "GPU_SyncFilm"}
    lib = ctypes.CDLL(LIB, mode=os.RTLD_LOCAL)
    for n in names:
        assert hasattr(lib, n), n
