"""The reference's PDRF bitwise grid (cpp/tests/pdrf_fusion_smoke.cu:57-88): a 19x17x13 field of
DBF / DAF values in [-2, 10) whose first 144 entries pair twelve special float32 bit patterns
(zeros, infinities, NaNs with payloads, denormals, the largest finite values, 1), under every
combination of the object's DBF maximum, its largest DAF, pdrf_scale and pdrf_exponent."""
import itertools

import numpy as np

SPECIAL = [0x00000000, 0x80000000, 0x7F800000, 0xFF800000, 0x7FC01234, 0xFFC04321,
           0x00000001, 0x80000001, 0x7F7FFFFF, 0xFF7FFFFF, 0x3F800000, 0x7F801234]
MAXIMA = [10.0, 0.0, 1e-30, 1e30, float("inf"), float("nan")]
MAX_DAFS = [10.0, 0.0, -0.0, 1e-300, float("inf"), float("nan")]
SCALES = [5000.0, 0.0, -1.0]
EXPONENTS = [1.0, 2.0, 4.0, 16.0, 0.0, -1.0, 2.5, 65536.0]


def fields(seed=470):
    rng = np.random.default_rng(seed)
    n = 19 * 17 * 13
    dbf = rng.uniform(-2, 10, n).astype(np.float32)
    daf = rng.uniform(-2, 10, n).astype(np.float32)
    bits_d, bits_a = dbf.view(np.uint32), daf.view(np.uint32)
    for i, j in itertools.product(range(12), range(12)):
        bits_d[12 * i + j] = SPECIAL[i]
        bits_a[12 * i + j] = SPECIAL[j]
    return dbf, daf


def grid():
    return itertools.product(MAXIMA, MAX_DAFS, SCALES, EXPONENTS)


def power_of_two(exponent):
    return 0 < exponent < 65536 and float(exponent).is_integer() and (int(exponent) & (int(exponent) - 1)) == 0


def same(a, b):
    """Bitwise equal, except that any two NaNs are equal (payloads are not part of the rule)."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    both_nan = np.isnan(a) & np.isnan(b)
    return (a.view(np.uint32) == b.view(np.uint32)) | both_nan
