"""Measurement hooks of the library run and report sane values: the FP32 peak
probe and the hill-slice staging probe (16-byte cp.async against one bulk copy
per array, no multicast) on the 64-walker workload's table size."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_hill_staging_probe():
    from gluedmd_b200 import _native
    out = (ctypes.c_double * 2)()
    st = ctypes.c_int(-1)
    _native.call("glued_measure_hill_staging", 50000, 148, 5, out, ctypes.byref(st))
    assert st.value == 0
    assert 0.5 < out[0] < 1000 and 0.5 < out[1] < 1000, (out[0], out[1])


def test_hill_staging_probe_rejects_oversize_slices():
    from gluedmd_b200 import _native, GluedError
    out = (ctypes.c_double * 2)()
    st = ctypes.c_int(0)
    with pytest.raises(GluedError):
        _native.call("glued_measure_hill_staging", 100000, 148, 1, out, ctypes.byref(st))


def test_fp32_peak_probe():
    from gluedmd_b200 import _native
    t = ctypes.c_double()
    _native.call("glued_measure_fp32_peak", ctypes.byref(t))
    assert 20.0 < t.value < 200.0
