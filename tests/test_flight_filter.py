"""The premises of the trackers' free-flight exit filter.

A Woodcock free flight t' = t - log(1 - u) / majorant * dt * w2g (deviceCode.cu:805, 915)
that certainly leaves the current cell is decided from the hardware log2 with a margin;
only the other flights run the exact chain of the arithmetic specification.  The margin
holds when (a) the project log is within 1.6e-7 (relative) of the true log on every
argument a flight takes, x = 1 - k 2^-24 for k < 2^24, and non-increasing in k, and (b)
the hardware log2 is within 2^-20 * (1 + |log2 x|) of log2 x on the same arguments; the
kernels' margin constants are 2^-18, four times (b) and more than twenty times (a).
Whether the filter changes any result is what every GPU parity test checks: the frames
stay bit-identical to the oracle's.
"""
import ctypes as C

import pytest


def test_project_log_bound_over_every_flight_argument(oracle):
    lib = oracle.load_oracle()
    lib.orc_flight_log_bound.restype = C.c_double
    lib.orc_flight_log_bound.argtypes = [C.POINTER(C.c_uint64)]
    up = C.c_uint64(0)
    worst = lib.orc_flight_log_bound(C.byref(up))
    assert worst <= 1.6e-7, worst
    assert up.value == 0


def test_quotient_from_the_stored_reciprocal_is_the_ieee_quotient(oracle):
    """The trackers divide by a majorant (and the TF remap by its spans) as q = RN(a y),
    RN(q + y (a - q b)) with the stored y = RN(1/b) (Markstein 1990): the same bits as the
    IEEE quotient, here over 64 M random pairs and every divisor mantissa x 16 dividends."""
    lib = oracle.load_oracle()
    lib.orc_quotient_check.restype = C.c_uint64
    lib.orc_quotient_check.argtypes = [C.c_uint64, C.c_int, C.c_uint64]
    assert lib.orc_quotient_check(64 << 20, 16, 12345) == 0


@pytest.mark.gpu
def test_hardware_log2_bound_over_every_flight_argument(mdwt_lib):
    worst = C.c_float(-1.0)
    mdwt_lib.mdwt_check_flight_filter.argtypes = [C.POINTER(C.c_float)]
    assert mdwt_lib.mdwt_check_flight_filter(C.byref(worst)) == 0
    assert 0.0 <= worst.value <= 2.0 ** -20, worst.value
