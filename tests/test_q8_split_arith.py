"""The integer forms of the 1/256 texel split the back projectors use, checked exhaustively
on the host against the split they replace (NumPy float32 / uint32 arithmetic; no GPU).

For a clamped texel coordinate c, q = floor(256 c - 127.5) sits in the mantissa of
f = 1.5 * 2^23 + q (bits = 0x4B400000 + q for |q| < 2^22).  The reference's split
(split_coord: texel floor(q / 256), weight (q mod 256) / 256) is then formed as

* shift and mask-or (column and fused SART kernels): (bits >> 8) - 0x4B4000 and
  float(((bits << 15) & 0x7F8000) | 0x3F800000) - 1;
* byte permute (perspective kernel): float(0x3F800000 | (bits & 255) << 8) * 128 - 128,
  with one rounding as a fused multiply-add (the product is exact in float64 here), and the
  texel index (bv >> 8) * pitch + (bu >> 8) - 0x4B4000 (pitch + 1) in wrapping 32-bit
  arithmetic.
"""
import numpy as np

C = 0x4B400000


def _bits(q):
    return (np.int64(C) + np.asarray(q, np.int64)).astype(np.uint32)


def test_bits_hold_q():
    q = np.arange(-2048, 1 << 21, dtype=np.int64)
    f = np.float32(12582912.0) + q.astype(np.float32)  # exact: |q| < 2^22
    assert np.array_equal(f.view(np.uint32), _bits(q))


def test_shift_mask_split_equals_floor_split():
    q = np.arange(-2048, 1 << 20, dtype=np.int64)
    b = _bits(q)
    x0 = (b.astype(np.int64) >> 8) - (C >> 8)
    a1 = (((b.astype(np.uint32) << np.uint32(15)) & np.uint32(0x7F8000)) | np.uint32(0x3F800000)).view(np.float32)
    a = a1 - np.float32(1.0)
    assert np.array_equal(x0, np.floor_divide(q, 256))
    assert np.array_equal(a, (np.mod(q, 256) / 256.0).astype(np.float32))


def test_byte_permute_weight_equals_floor_split():
    q = np.arange(-2048, 1 << 20, dtype=np.int64)
    b = _bits(q)
    k1 = (np.uint32(0x3F800000) | ((b & np.uint32(0xFF)) << np.uint32(8))).view(np.float32)
    # fma(k1, 128, -128): the exact value rounded once (float64 holds it exactly)
    w = (k1.astype(np.float64) * 128.0 - 128.0).astype(np.float32)
    assert np.array_equal(w, (np.mod(q, 256) / 256.0).astype(np.float32))


def test_folded_texel_index_equals_row_major_index():
    rng = np.random.Generator(np.random.PCG64(5))
    for pitch in (16, 1028, 2056, 4100):
        qu = rng.integers(-512, (pitch - 4) * 256, 200000)
        qv = rng.integers(-512, 2000 * 256, 200000)
        bu, bv = _bits(qu), _bits(qv)
        kq = np.uint32((0x4B4000 * (pitch + 1)) & 0xFFFFFFFF)
        with np.errstate(over="ignore"):
            t = ((bv >> np.uint32(8)) * np.uint32(pitch) + (bu >> np.uint32(8)) - kq).view(np.int32)
        want = np.floor_divide(qv, 256) * pitch + np.floor_divide(qu, 256)
        assert np.array_equal(t.astype(np.int64), want)
