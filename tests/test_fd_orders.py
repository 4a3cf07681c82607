"""Corrector orders (host logic, no GPU): the reference's coefficient sets (FSLBM.cu:177-232)
as the library and the oracle hold them."""
import numpy as np
import pytest

import oracle_lib as O

ORDERS = [(0, 0.0), (4, 1.0), (6, 0.4), (6, 1.0), (8, 0.5), (8, 1.0), (10, 0.0), (12, 0.0), (14, 0.0)]


@pytest.mark.parametrize("order,blend", ORDERS)
def test_library_and_oracle_tables_agree(built, order, blend):
    lib64 = built.fd_coefficients(order, blend, built.F64)
    assert np.array_equal(lib64, O.fd_coefficients(order, blend))
    # FP32 solves form the coefficients in FP32 as the reference does (FSLBM.cu:231)
    lib32 = built.fd_coefficients(order, blend, built.F32)
    assert lib32.dtype == np.float64 and np.all(lib32 == lib32.astype(np.float32))
    assert np.allclose(lib32, lib64, rtol=1e-6, atol=1e-9)


def test_fp32_forms_follow_the_reference_arithmetic(built):
    b = np.float32(0.4)
    c = built.fd_coefficients(6, 0.4, built.F32)
    assert c[0] == np.float32(np.float32(-7.5) - np.float32(0.66666666666) * b)
    assert c[3] == np.float32(np.float32(0.01111111) * b)


@pytest.mark.parametrize("order,blend,want", [(4, 1.0, 6), (6, 1.0, 8), (8, 1.0, 10), (10, 0.0, 12),
                                              (12, 0.0, 14), (14, 0.0, 16), (0, 0.0, 4), (6, 0.4, 6)])
def test_consistency_and_order(order, blend, want):
    """Per axis the corrector's symbol sum_k c_k 2(cos k t - 1) approximates -t^2 with an error
    of order t^(N+2) for the nominal order N (blends: the lower order's), and c0 + 6 sum c_k = 0
    to the precision of the reference's decimals."""
    c = O.fd_coefficients(order, blend)
    assert abs(c[0] + 6 * c[1:].sum()) <= 2e-7 * abs(c[0])
    k = np.arange(1, len(c))
    err = lambda t: np.sum(c[1:] * 2 * (np.cos(k * t) - 1)) + t * t
    observed = np.log2(abs(err(1.0) / err(0.5)))
    assert observed >= want - 0.7, observed


def test_unknown_order_rejected(built):
    with pytest.raises(built.FslbmError):
        built.fd_coefficients(5)
    with pytest.raises(ValueError):
        O.fd_coefficients(16)
