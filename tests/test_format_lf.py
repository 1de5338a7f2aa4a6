"""The text writer's "%lf" formatter (felog_format_lf) against correctly
rounded decimal conversion (Python's '%f', which glibc's printf agrees with):
random magnitudes, exact ties (odd multiples of 2^-7 .. 2^-20 round half to
even), BF16-valued floats, subnormals, signed zeros and infinities."""
import numpy as np

import felog_b200 as fb


def check(vals):
    vals = np.asarray(vals, np.float32)
    got = fb.format_lf(vals).split(" ")[:-1]
    want = ["%f" % float(v) for v in vals]
    bad = [(float(v), g, w) for v, g, w in zip(vals, got, want) if g != w]
    assert not bad, bad[:10]


def test_random_magnitudes():
    rng = np.random.default_rng(7)
    check(rng.uniform(-1, 1, 200000))
    check(rng.standard_normal(100000) * 10.0 ** rng.integers(-9, 12, 100000))
    check(rng.lognormal(0, 8, 50000) * rng.choice([-1, 1], 50000))


def test_ties_round_half_even():
    j = np.arange(-4097, 4098, 2, dtype=np.float64)
    for k in range(7, 21):
        check(j / 2.0 ** k)
    check([0.0078125, -0.0078125, 0.0234375, 1.0000005 - 0.0000005 + 0.0078125])


def test_bf16_values_and_special():
    rng = np.random.default_rng(3)
    h = rng.integers(0, 1 << 16, 100000, dtype=np.uint32) << 16
    v = h.view(np.float32)
    check(v[np.isfinite(v)])
    sub = (rng.integers(1, 1 << 23, 1000, dtype=np.uint32)).view(np.float32)
    check(sub)
    check([0.0, -0.0, np.inf, -np.inf, 1e-45, -1e-45, 3.4028235e38, -3.4028235e38, 2.0 ** 40, 2.0 ** 39 + 0.5])
