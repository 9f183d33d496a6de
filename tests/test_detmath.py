"""Deterministic transcendental functions (include/vxe/detmath.h) against float64 numpy."""
import numpy as np

from oracle import oracle as O


def ulp_err(got, ref64):
    got = got.astype(np.float64)
    ref32 = ref64.astype(np.float32)
    spacing = np.spacing(np.abs(ref32)).astype(np.float64)
    return np.abs(got - ref64) / np.maximum(spacing, np.finfo(np.float32).tiny)


def test_sin_cos_within_one_and_a_half_ulp():
    rng = np.random.default_rng(1)
    # binary32 path (|x| <= 65536) and the binary64 reduction beyond it
    x = np.concatenate([rng.uniform(-10, 10, 200000), rng.uniform(-65536, 65536, 200000),
                        rng.uniform(-5e5, 5e5, 50000)]).astype(np.float32)
    for which, fn in ((0, np.sin), (1, np.cos)):
        got = O.detmath(which, x)
        ref = fn(x.astype(np.float64))
        # near the zeros of sin/cos the error is measured in absolute terms
        err = np.abs(got.astype(np.float64) - ref)
        assert (err <= np.maximum(1.5 * np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64), 8e-8)).all()


def test_exp_within_one_ulp():
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-80, 80, 200000), rng.uniform(-1, 1, 100000),
                        rng.uniform(-103, -87, 50000)]).astype(np.float32)
    got = O.detmath(2, x)
    assert ulp_err(got, np.exp(x.astype(np.float64))).max() <= 1.0


def test_pow_error_bounds_for_shader_exponents():
    # binary32 throughout: 1.25 ulp for exponents up to 8; the error grows
    # with |y log x| (3.5 ulp at 96)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.0, 1.0, 200000).astype(np.float32)
    for e in (0.98, 1.0 / 2.2, 0.5, 1.5, 1.6, 1.8, 2.0, 2.4, 3.0, 5.0, 8.0, 96.0):
        y = np.full_like(x, np.float32(e))
        got = O.detmath(3, x, y)
        ref = np.power(x.astype(np.float64), np.float64(np.float32(e)))
        ok = ulp_err(got, ref) <= (1.25 if e <= 8.0 else 3.5)
        ok |= np.abs(got.astype(np.float64) - ref) < 1e-38  # underflow region
        assert ok.all(), e
    assert O.detmath(3, np.array([0.0, 1.0, 0.0], np.float32), np.array([2.0, 7.0, 0.0], np.float32)).tolist() == [
        0.0, 1.0, 1.0]


def test_special_values():
    nan = np.float32(np.nan)
    s = O.detmath(0, np.array([np.inf, nan, 0.0, -0.0], np.float32))
    assert np.isnan(s[0]) and np.isnan(s[1]) and s[2] == 0.0
    e = O.detmath(2, np.array([-200.0, 100.0, 0.0], np.float32))
    assert e[0] == 0.0 and np.isinf(e[1]) and e[2] == 1.0
    # min/max: NaN-ignoring, -0 < +0 (IEEE minimumNumber / maximumNumber)
    mn = O.detmath(4, np.array([nan, 1.0, 0.0, -0.0], np.float32), np.array([2.0, nan, -0.0, 0.0], np.float32))
    assert mn[0] == 2.0 and mn[1] == 1.0 and np.signbit(mn[2]) and np.signbit(mn[3])
    mx = O.detmath(5, np.array([0.0, -0.0], np.float32), np.array([-0.0, 0.0], np.float32))
    assert not np.signbit(mx[0]) and not np.signbit(mx[1])
