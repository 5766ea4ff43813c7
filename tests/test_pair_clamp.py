"""The FP32 near field's pair weight, restated on the CPU.

The tensor-core form's near field (csrc/fmm_tc.cu, tc_pair2) evaluates
d3's pair formula (many_body.zig:176-263: w = s / l, or s / sqrt(dmin2 l)
inside distanceMin) as w = s * rsqrt(y). Its scalar form took
y = lf max(lf, dmin2) with lf = max(l, 1e-18). The packed form takes
y = max(l^2, l dmin2, fl) with fl = 1e-18 max(1e-18, dmin2), so that both
halves of a packed pair need only multiplies and maxima. Rounding is
monotonic, so the two are equal bit for bit in FP32. This test checks that
over a log-uniform spread of squared distances (tiny and huge ones
included) and the distanceMin values in use, 0 among them.
"""

import numpy as np
import pytest

F = np.float32
FLOOR = F(1e-18)


def _y_scalar(l, d):
    lf = np.maximum(l, FLOOR)
    return lf * np.maximum(lf, d)


def _y_packed(l, d):
    fl = FLOOR * np.maximum(FLOOR, d)
    return np.maximum(np.maximum(l * l, l * d), fl)


@pytest.mark.parametrize("dmin", [0.0, 1e-6, 0.5, 1.0, 2.0, 30.0, 1e4])
def test_packed_clamp_equals_scalar_clamp(dmin):
    rng = np.random.default_rng(17)
    d = F(dmin) * F(dmin)
    l = (10.0 ** rng.uniform(-40, 30, 200000)).astype(F)
    special = np.array([0.0, FLOOR, np.nextafter(FLOOR, F(0)), np.nextafter(FLOOR, F(1)), d,
                        np.nextafter(d, F(0)), np.nextafter(d, F(np.inf)), 1.0, 1e-30, 1e19],
                       dtype=F)
    l = np.concatenate([l, special])
    with np.errstate(over="ignore", under="ignore"):
        a, b = _y_scalar(l, d), _y_packed(l, d)
    assert a.dtype == F and b.dtype == F
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # the self pair (l = 0) keeps a finite weight, so 0 * w adds nothing
    assert np.isfinite(1.0 / np.sqrt(b[l == 0])).all()
