"""The oracle's weighted back projection (WBP plugin, plugins/WBPPlugin/src/reconstruction/
WBP.cpp): the RamLak filtering restated from ConvolutionFourierSpaceImplementation (FFT on
the power-of-two grid) against a direct circular convolution of the same padded grid, the
one-row displacement of the filtered image that the kernel's origin move produces, and,
where the reference checkout is present, the reference's own WBP test
(WBPPluginTest.cpp Integration: max slice RMS < 0.05 against its ground_truth.mrc).
Host only."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import reference_path

REF_WBP = reference_path("ettention", "plugins", "WBPPlugin", "test", "data", "wbp_shepp_logan")


def _direct_filter(img, fres=128):
    """Circular convolution on the padded grid, written out: padded row y + 1 (mod Hu) for
    an even Hu, taps at positions p = -fres/2 .. fres/2 - 1, centred crop."""
    H, W = img.shape
    Wu, Hu = O._next_pow2(max(W, fres)), O._next_pow2(H)
    src = np.asarray(img, np.float64)[O._pad_index(np.arange(Hu), H, Hu)][:, O._pad_index(np.arange(Wu), W, Wu)]
    k = O.ramlak_kernel(fres).astype(np.float64)
    out = np.zeros((Hu, Wu))
    dy = 1 if Hu > 1 else 0
    for g in range(fres):
        p = g - fres // 2
        out += k[g] * np.roll(np.roll(src, -dy, axis=0), p, axis=1)
    cx, cy = Wu // 2 - W // 2, Hu // 2 - H // 2
    return out[cy:cy + H, cx:cx + W].astype(np.float32)


def test_ramlak_kernel_values():
    k = O.ramlak_kernel(128)
    assert k[64] == np.float32(0.25)
    assert k[65] == k[63] and k[66] == 0 and k[0] == 0
    assert np.isclose(k[65], -1 / np.pi ** 2, rtol=1e-6) and np.isclose(k[67], -1 / (9 * np.pi ** 2), rtol=1e-6)


def test_filter_rejects_images_the_mirrored_padding_would_leave():
    with pytest.raises(ValueError, match="leaves the image"):
        O.wbp_filter(np.zeros((7, 5), np.float32))  # 5 columns padded to 128


@pytest.mark.parametrize("shape", [(64, 128), (30, 100), (1, 256), (130, 300), (3, 50)])
def test_fft_filter_equals_direct_circular_convolution(shape):
    img = np.random.default_rng(shape[0] * 1000 + shape[1]).standard_normal(shape).astype(np.float32)
    a = O.wbp_filter(img)
    b = _direct_filter(img)
    assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()


def test_filter_of_a_delta_is_the_kernel_one_row_up():
    img = np.zeros((64, 128), np.float32)
    img[20, 40] = 1.0
    f = O.wbp_filter(img)
    k = O.ramlak_kernel(128)
    want = np.zeros_like(f)
    for g in range(128):
        want[19, (40 + g - 64) % 128] = k[g]
    assert np.abs(f - want).max() <= 1e-7


@pytest.mark.skipif(not os.path.isdir(REF_WBP), reason="ETTENTION_REFERENCE (reference checkout) not set")
def test_oracle_wbp_meets_the_reference_test_bound():
    from ettention_b200.operators import MRCStack
    s = MRCStack(os.path.join(REF_WBP, "empiar_10009_128.mrc"), os.path.join(REF_WBP, "empiar_10009_128.tlt"))
    vg = O.VolumeGeometry.centered((128, 128, 20))
    base = O.mrc_base_geometry(128, 128)
    v = O.wbp(s.load_projections(), [O.rotate_geometry(base, float(a)) for a in s.tilt_angles], vg)
    gt = MRCStack(os.path.join(REF_WBP, "ground_truth.mrc")).load_projections()  # xyz_order: (z, y, x)
    assert O.max_slice_rms(v, gt) < 0.05  # WBPPluginTest.cpp Integration
