"""Seeded synthetic posit32 inputs shaped like the benchmark configurations.

The generators follow the configurations' stated distributions: entries uniform in
[-1, 1] (FP64, then converted to posit32), or a wide-dynamic-range variant with
magnitudes 10^U(-20, 20) and random signs.  Conversion is the oracle's correctly
rounded one, so the GPU and the oracle always see the same bit patterns.
"""
import numpy as np

import oracle


def uniform(rng, shape):
    return oracle.from_double(rng.uniform(-1.0, 1.0, size=shape))


def wide(rng, shape):
    mag = 10.0 ** rng.uniform(-20.0, 20.0, size=shape)
    sign = np.where(rng.integers(0, 2, size=shape) == 1, -1.0, 1.0)
    return oracle.from_double(sign * mag)


def colmajor(rng, rows, cols, ld=None, kind="uniform"):
    """Flat column-major buffer of ld*cols posit32 (rows beyond `rows` hold junk)."""
    ld = ld or rows
    gen = uniform if kind == "uniform" else wide
    buf = gen(rng, (ld * cols,))
    return buf
