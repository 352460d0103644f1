"""SIMT arithmetic peaks measured by the library's microbenchmark (rt_bench_simt_peak): the
numbers the bench sets the matrix-free finest-level kernel against.  Plausibility bounds only:
FP32 (scalar and packed FFMA2) above 20 TFLOP/s and FP64 above 5 TFLOP/s on a B200, and every
figure below 200 TFLOP/s (a timing that skipped work).  The packed form is not required to beat
the scalar one: on B200 it measured below it."""
import ctypes as C

import pytest

import robtop_b200 as rb

pytestmark = pytest.mark.gpu


def test_simt_peaks_plausible():
    ctx = rb.Context(0)
    try:
        vals = []
        for kind in (0, 1, 2):
            t = C.c_double()
            rb._capi.check(rb.lib().rt_bench_simt_peak(ctx.handle, kind, 3, C.byref(t)), ctx.handle)
            vals.append(t.value)
        fp32, fp32x2, fp64 = vals
        assert 20 < fp32 < 200 and 20 < fp32x2 < 200 and 5 < fp64 < 200
        assert rb.lib().rt_bench_simt_peak(ctx.handle, 3, 1, C.byref(C.c_double())) != 0
    finally:
        ctx.close()
