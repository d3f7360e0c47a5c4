"""The CNN oracle (oracle/cnn.py) pinned on the CPU: BF16 rounding against
known bit patterns, the 3x3 convolution against direct loops, and the two
gradient identities the GPU tests rely on -- the data gradient is the
convolution with flipped, transposed weights (adjointness) and the weight
gradient is the derivative of <conv(x, w), y> in w."""
import numpy as np

from oracle import cnn as ocnn


def test_bf16_rounds_to_nearest_even():
    ulp = 2.0 ** -7  # bfloat16 spacing at 1.0 (7 stored mantissa bits)
    cases = [
        (1.0, 1.0),
        (1.0 + ulp / 2, 1.0),                 # tie, even neighbour below
        (1.0 + 1.5 * ulp, 1.0 + 2 * ulp),     # tie, even neighbour above
        (1.0 + ulp / 2 + 2.0 ** -20, 1.0 + ulp),
        (-(1.0 + 1.5 * ulp), -(1.0 + 2 * ulp)),
    ]
    for v, want in cases:
        assert ocnn.bf16(np.float32(v)) == np.float32(want), v
    assert ocnn.bf16_bits(np.float32(1.0)) == 0x3F80
    assert ocnn.bf16_bits(np.float32(-2.0)) == 0xC000
    # random magnitudes: the nearer of the two bf16 neighbours, ties to the even one
    rng = np.random.default_rng(6)
    v = (rng.standard_normal(4096) * 10.0 ** rng.integers(-30, 30, 4096)).astype(np.float32)
    bits = v.view(np.uint32).astype(np.uint64)
    lo = (bits & 0xFFFF0000).astype(np.uint32).view(np.float32).astype(np.float64)
    hi = ((bits & 0xFFFF0000) + 0x10000).astype(np.uint32).view(np.float32).astype(np.float64)
    d_lo, d_hi = np.abs(v - lo), np.abs(hi - v)
    lo_even = ((bits >> 16) & 1) == 0
    want = np.where((d_lo < d_hi) | ((d_lo == d_hi) & lo_even), lo, hi).astype(np.float32)
    np.testing.assert_array_equal(ocnn.bf16(v), want)


def _direct_conv(x, w, b):
    B, H, W, CI = x.shape
    CO = w.shape[0]
    out = np.zeros((B, H, W, CO))
    for n in range(B):
        for y in range(H):
            for xx in range(W):
                for co in range(CO):
                    s = b[co]
                    for t in range(9):
                        dy, dx = divmod(t, 3)
                        yy, xs = y + dy - 1, xx + dx - 1
                        if 0 <= yy < H and 0 <= xs < W:
                            s += float(np.dot(w[co, t], x[n, yy, xs]))
                    out[n, y, xx, co] = s
    return out


def test_conv3x3_matches_direct_loops_with_zero_padding():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, 3, 5, 4))
    w = rng.standard_normal((3, 9, 4))
    b = rng.standard_normal(3)
    np.testing.assert_allclose(ocnn.conv3x3(x, w, b), _direct_conv(x, w, b), rtol=0, atol=1e-12)


def test_data_gradient_is_the_flipped_transposed_convolution():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((2, 6, 7, 4))
    y = rng.standard_normal((2, 6, 7, 5))
    w = rng.standard_normal((5, 9, 4))
    lhs = float(np.sum(ocnn.conv3x3(x, w) * y))
    rhs = float(np.sum(x * ocnn.conv3x3(y, ocnn.flip_transpose(w))))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_weight_gradient_is_the_derivative_in_the_weights():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, 6, 7, 4))
    y = rng.standard_normal((2, 6, 7, 5))
    w = rng.standard_normal((5, 9, 4))
    # <conv(x, w), y> is linear in w, so it equals <w, dW> with dW the gradient
    lhs = float(np.sum(ocnn.conv3x3(x, w) * y))
    rhs = float(np.sum(w * ocnn.conv_wgrad(y, x)))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
