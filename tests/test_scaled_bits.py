"""The loss kernels build H's FP64 values from the float bits with integer
operations (f32_scaled in kernels_loss.cu): the 8-bit exponent field and the
23-bit fraction move into the low bits of the double's exponent field and
the top of its fraction, which reads as f * 2^-896 for every finite float,
subnormals and zeros included.  This checks that construction, restated in
numpy, on every class of float."""
import numpy as np


def scaled_bits(f):
    b = f.view(np.uint32).astype(np.uint64)
    hi = ((b >> np.uint64(3)) & np.uint64(0x0FFFFFFF)) | (b & np.uint64(0x80000000))
    lo = (b << np.uint64(29)) & np.uint64(0xFFFFFFFF)
    return ((hi << np.uint64(32)) | lo).view(np.float64)


def test_scaled_bits_is_f_times_2_to_minus_896():
    rng = np.random.default_rng(0)
    parts = [
        np.array([0.0, -0.0, 1.0, -1.0, 2.0 ** -126, 2.0 ** -149, -(2.0 ** -149),
                  np.finfo(np.float32).max, -np.finfo(np.float32).max], np.float32),
        rng.standard_normal(100_000).astype(np.float32),
        (rng.uniform(-1, 1, 100_000) * 2.0 ** -130).astype(np.float32),  # subnormal floats
        rng.integers(0, 0x7F800000, 100_000, dtype=np.uint32).view(np.float32),  # any finite
    ]
    f = np.concatenate(parts)
    got = scaled_bits(f)
    want = f.astype(np.float64) * 2.0 ** -896
    np.testing.assert_array_equal(got, want)
    # scaled back by the power of two, exactly the float's value
    np.testing.assert_array_equal(got * 2.0 ** 896, f.astype(np.float64))


def test_scaled_products_round_as_unscaled():
    # a sum of products formed at scale 2^-896 and scaled back equals the
    # unscaled FP64 sum while the scaled terms stay normal doubles
    rng = np.random.default_rng(1)
    w = rng.standard_normal((1000, 32)).astype(np.float32)
    h = rng.standard_normal((1000, 32)).astype(np.float32)
    plain = np.zeros(1000)
    scaled = np.zeros(1000)
    hs = scaled_bits(h.ravel()).reshape(h.shape)
    for z in range(32):  # the kernel's order: one accumulator, z ascending
        plain = plain + w[:, z].astype(np.float64) * h[:, z].astype(np.float64)
        scaled = scaled + w[:, z].astype(np.float64) * hs[:, z]
    np.testing.assert_array_equal(scaled * 2.0 ** 896, plain)
