"""crmath.cuh on the host (through the oracle library, which compiles the same
header): sin/cos correctly rounded, checked against 40-digit decimal
arithmetic; the platform libm (glibc, the reference's) agrees except in a
small fraction of its results, which is what the terrain-correction parity
tests exclude when they compare against the glibc oracle.
The device copy is compared bit for bit with this one in test_gpu_tc.py."""
from decimal import Decimal, getcontext
import math

import numpy as np

import oracle


def _pi():
    getcontext().prec = 45

    def atan_inv(n):
        x = Decimal(1) / n
        s, t, k = Decimal(0), x, 1
        while abs(t / k) > Decimal(10) ** -44:
            s += t / k if (k // 2) % 2 == 0 else -t / k
            t *= x * x
            k += 2
        return s
    return 16 * atan_inv(5) - 4 * atan_inv(239)


PI = _pi()


def _sin_cos_exact(x: float):
    """sin and cos of the double x to ~1e-40, rounded to the nearest double."""
    getcontext().prec = 45
    d = Decimal(x)  # exact value of the double
    k = int((d / (PI / 2)).to_integral_value())
    r = d - k * (PI / 2)
    s, c, t, n = Decimal(0), Decimal(0), Decimal(1), 0
    while abs(t) > Decimal(10) ** -44 or n < 2:
        if n % 4 == 0:
            c += t
        elif n % 4 == 1:
            s += t
        elif n % 4 == 2:
            c -= t
        else:
            s -= t
        n += 1
        t = t * r / n
    s, c = [(s, c), (c, -s), (-s, -c), (-c, s)][k % 4]
    return float(s), float(c)


def test_cr_sincos_is_correctly_rounded():
    rng = np.random.default_rng(5)
    x = np.concatenate([
        rng.uniform(-math.pi, math.pi, 1500),        # latitudes and longitudes in radians
        rng.uniform(0.6, 1.0, 600),                   # mid-latitudes
        rng.uniform(-10.0, 10.0, 400),                # Lanczos-3 arguments
        rng.uniform(-1e-3, 1e-3, 200),
        rng.uniform(-1e5, 1e5, 200),
        np.array([0.0, -0.0, 1e-300, 5e-324, math.pi / 2, math.pi, 3 * math.pi / 2, 2 * math.pi,
                  math.pi / 4, np.nextafter(math.pi / 4, 1.0), 1e-8, 0.5, 1.0]),
    ])
    s, c = oracle.cr_sincos(x)
    bad = []
    for xi, si, ci in zip(x, s, c):
        es, ec = _sin_cos_exact(float(xi))
        if si != es or ci != ec:
            bad.append((float(xi).hex(), si, es, ci, ec))
    assert not bad, bad[:5]


def test_glibc_disagrees_with_correct_rounding_rarely():
    rng = np.random.default_rng(6)
    x = rng.uniform(0.2, 1.4, 200_000)
    s, c = oracle.cr_sincos(x)
    n_bad = int((np.sin(x) != s).sum() + (np.cos(x) != c).sum())
    # a few in a thousand: the pixels where the reference's own libm and a
    # correctly rounded one disagree
    assert 0 <= n_bad <= 0.01 * 2 * x.size


def test_libm_switch_restores_and_changes_only_libm_pixels():
    """The oracle's libm setting is scoped, and the two settings give the same
    geocoding except at a few pixels."""
    from sardine_b200 import synth
    sc = synth.config1_scene(seed=8, n_lines=256, n_samples=512, dem_n=96, flatten=True)
    gl = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    with oracle.libm("cr"):
        assert oracle.lib().orc_get_libm() == 1
        cr = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    assert oracle.lib().orc_get_libm() == 0
    same = (gl.data == cr.data) | (np.isnan(gl.data) & np.isnan(cr.data))
    assert same.mean() > 0.99
    assert np.array_equal(gl.mask, cr.mask) or (gl.mask != cr.mask).mean() < 1e-3
