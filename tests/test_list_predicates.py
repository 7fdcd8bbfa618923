"""The FP32 predicates of the neighbour-list kernels, checked on the CPU with
numpy float32 arithmetic (IEEE round to nearest, as the device's FP32 adds).

- k_list_scan tests 0 < r^2 < R^2 as one unsigned compare of the bit
  patterns, bits(r^2) - 1 < bits(R^2) - 1: equal to the two float compares
  for every non-negative float (r^2 is a sum of squares).
- The half2 list pass sends an entry to the FP32 record when
  |(|r^2 - H2/2|) - H2/2| < band (H2 = (2h)^2): r^2 within the band of 0 or
  of H2.  Its two roundings are at most ulp(H2) / 4 each, and the band carries
  a margin of 16 ulp(H2) (h16_band in csrc/sim.cu), so every r^2 within the
  band less that margin of 0 or of H2 is flagged."""
import numpy as np

f32 = np.float32


def unsigned_test(r2, bound):
    b = np.asarray(r2, np.float32).view(np.uint32)
    hb = np.uint32(np.float32(bound).view(np.uint32)) - np.uint32(1)
    return (b - np.uint32(1)) < hb  # uint32 wraps 0 - 1 to 0xffffffff


def float_test(r2, bound):
    r2 = np.asarray(r2, np.float32)
    return (r2 > f32(0)) & (r2 < f32(bound))


def test_unsigned_compare_equals_the_float_compares():
    rng = np.random.default_rng(0)
    for bound in (f32(1.69e-4), f32(0.0213), f32(1.0), f32(3.3e-9), f32(7.5e5)):
        r2 = np.concatenate([
            rng.uniform(0.0, 4.0 * float(bound), 200000).astype(np.float32),
            np.array([0.0, np.finfo(np.float32).tiny, 1e-45, float(bound)], np.float32),
            np.nextafter(bound, f32(0), dtype=np.float32)[None],
            np.nextafter(bound, f32(np.inf), dtype=np.float32)[None],
            np.array([np.inf, 3.0e38], np.float32),
        ])
        np.testing.assert_array_equal(unsigned_test(r2, bound), float_test(r2, bound))


def folded_band(r2, h2, band):
    r2 = np.asarray(r2, np.float32)
    hm = f32(0.5) * f32(h2)
    return np.abs(np.abs(r2 - hm) - hm) < f32(band)


def test_folded_band_covers_both_ends():
    for h2 in (f32(1.69e-4), f32(6.76e-4), f32(0.0213), f32(2.7e-6)):
        ulp = np.nextafter(h2, f32(np.inf), dtype=np.float32) - h2
        margin = f32(16) * ulp
        for band in (f32(2e-4) * h2 + margin, f32(1e-5) * h2 + margin, f32(64) * ulp):
            inner = float(band) - float(margin)
            near0 = np.linspace(0.0, inner * (1 - 1e-6), 20001).astype(np.float32)
            nearH = (float(h2) + np.linspace(-inner, inner, 40001) * (1 - 1e-6)).astype(np.float32)
            assert folded_band(near0, h2, band).all()
            assert folded_band(nearH, h2, band).all()
            # and nothing far from both ends is flagged
            mid = np.linspace(2.0 * float(band), float(h2) - 2.0 * float(band), 20001).astype(np.float32)
            far = np.linspace(float(h2) + 2.0 * float(band), 4.0 * float(h2), 20001).astype(np.float32)
            assert not folded_band(mid, h2, band).any()
            assert not folded_band(far, h2, band).any()
