"""NumPy restatement of the e3m12 storage format (include/lbm_b200.h, LBM_DTYPE_E3M12) for tests:
sign, 3 exponent and 12 mantissa bits of value * 16; the codes are the bits of the FP32 number
value * 2^-115 shifted right by 11, rounded to nearest even, clamped to the largest finite code."""
import numpy as np


def encode(v):
    t = np.asarray(v, np.float32) * np.float32(2.0 ** -115)      # IEEE: subnormal results kept
    b = t.view(np.uint32)
    mag = b & np.uint32(0x7FFFFFFF)
    c = np.minimum((mag + np.uint32(0x3FF) + ((mag >> np.uint32(11)) & np.uint32(1))) >> np.uint32(11),
                   np.uint32(0x7FFF))
    return (c | ((b >> np.uint32(16)) & np.uint32(0x8000))).astype(np.uint16)


def decode(h):
    h = np.asarray(h).view(np.uint16).astype(np.uint32)
    b = ((h & np.uint32(0x7FFF)) << np.uint32(11)) | ((h & np.uint32(0x8000)) << np.uint32(16))
    return b.view(np.float32) * np.float32(2.0 ** 115)
