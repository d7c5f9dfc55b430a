"""The PDRF arithmetic over the reference's bitwise grid (cpp/tests/pdrf_fusion_smoke.cu:57-88):
the engine's own device arithmetic (brook_pdrf_values) against the oracle's restatement, bit for
bit where the power is repeated squaring and within float32 rounding of powf elsewhere; the oracle
alone on CPU."""
import numpy as np
import pytest

from oracle import oracle
from pdrf_grid import fields, grid, power_of_two, same


def test_oracle_grid_known_values():
    dbf, daf = fields()
    d = np.array([0.0, 2.0, 5.0], np.float32)
    a = np.array([np.inf, 3.0, 20.0], np.float32)
    out = oracle.pdrf_values(d, a, 10.0, 20.0, 5000.0, 2.0)
    m = np.float32(1.0 / 10.0 ** 1.01)
    p1 = np.float32(np.float32(1) - np.float32(2.0) * m)
    exp1 = np.float32(np.float32(p1 * p1) * np.float32(5000)) + np.float32(3.0) * np.float32(1 / 20.0)
    assert np.isinf(out[0]) and out[0] > 0   # a DBF of 0 counts as +inf: (1 - inf)^2 * 5000
    assert out[1] == exp1
    for maximum, max_daf, scale, exponent in grid():
        oracle.pdrf_values(dbf, daf, maximum, max_daf, scale, exponent)


@pytest.mark.gpu
def test_engine_pdrf_matches_the_grid(gpu):
    from brook_b200 import _native

    lib, ctx = _native.load(), _native.context(0)
    dbf, daf = fields()
    out = np.empty_like(dbf)
    checks = 0
    for maximum, max_daf, scale, exponent in grid():
        _native.check(lib.brook_pdrf_values(ctx, dbf.ctypes.data, daf.ctypes.data, dbf.size, maximum, max_daf, scale,
                                            exponent, out.ctypes.data))
        exp = oracle.pdrf_values(dbf, daf, maximum, max_daf, scale, exponent)
        ok = same(out, exp)
        if not power_of_two(exponent):
            # powf against float(pow(double)): equal up to a float32 rounding step of the power term
            # (scaled), which the DAF term can cancel down to a much smaller sum
            power = oracle.pdrf_values(dbf, daf, maximum, 0.0, scale, exponent)
            with np.errstate(invalid="ignore", over="ignore"):
                tol = (np.abs(power).astype(np.float64) + np.abs(exp)) * 2.0 ** -20
                close = np.abs(out.astype(np.float64) - exp.astype(np.float64)) <= tol
            ok |= np.isfinite(out) & np.isfinite(exp) & close
            ok |= np.isinf(out) & np.isinf(exp) & (np.sign(out) == np.sign(exp))
        bad = np.flatnonzero(~ok)
        assert bad.size == 0, (maximum, max_daf, scale, exponent, bad[:5], out[bad[:5]], exp[bad[:5]])
        checks += 1
    assert checks == 6 * 6 * 3 * 8
