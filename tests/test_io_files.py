"""File formats of the reconstruction's front door (host code, no GPU): MRC tilt
series in (modes 0 / 1 / 2 / 6, extended headers, MRCStack's log transform), tilt-angle
files, MRC volumes out in XYZ and XZY order.  The log transform is checked against a
NumPy restatement of MRCStack.cpp:161-172, 226-236; when the reference checkout is
present, its jason_64_SART stack and tilt file are read too."""
import os

import numpy as np
import pytest

from ettention_b200 import _abi
from ettention_b200._abi import EttentionError
from tests.helpers import reference_path

REF_DATA = reference_path("ettention", "test", "data", "jason_64_SART")


def write_stack(path, data, mode, extra=b""):
    """A 1024-byte MRC header (nx, ny, nz, mode, extended-header bytes) + data."""
    nz, ny, nx = data.shape
    h = np.zeros(256, np.int32)
    h[0], h[1], h[2], h[3] = nx, ny, nz, mode
    h[23] = len(extra)
    dtype = {0: np.uint8, 1: np.int16, 2: np.float32, 6: np.uint16}[mode]
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(extra)
        f.write(np.ascontiguousarray(data, dtype).tobytes())


def log_transform(raw, mode):
    """MRCStack: M = max - min + 1, m = min - 1 (modes 1, 2); M = max + 1, m = -1 (0, 6)."""
    r = raw.astype(np.float32)
    if mode in (1, 2):
        M, m = np.float32(r.max() - r.min() + 1), np.float32(r.min() - 1)
    else:
        M, m = np.float32(r.max() + 1), np.float32(-1.0)
    return np.log((M / (r - m)).astype(np.float32)).astype(np.float32)


@pytest.mark.parametrize("mode", [0, 1, 2, 6])
def test_stack_modes_extended_header_and_log_transform(tmp_path, mode):
    from ettention_b200.operators import MRCStack
    rng = np.random.Generator(np.random.PCG64(mode))
    if mode == 2:
        raw = rng.uniform(-3.0, 50.0, size=(5, 7, 9)).astype(np.float32)
    else:
        lo, hi = {0: (0, 255), 1: (-300, 3000), 6: (0, 60000)}[mode]
        raw = rng.integers(lo, hi, size=(5, 7, 9))
    path = tmp_path / "stack.mrc"
    write_stack(path, raw, mode, extra=bytes(range(256)) * 3)
    st = MRCStack(str(path))
    assert (st.info.nx, st.info.ny, st.info.nz, st.info.mode, st.info.extended_bytes) == (9, 7, 5, mode, 768)
    assert st.tilt_angles == [0.0] * 5
    assert np.array_equal(st.load_projections(), raw.astype(np.float32))
    lg = MRCStack(str(path), logarithmize=True).load_projections()
    np.testing.assert_allclose(lg, log_transform(raw, mode), rtol=2e-7, atol=1e-7)
    assert np.all(np.isfinite(lg))


def test_unsupported_mode_and_missing_file(tmp_path):
    from ettention_b200.operators import MRCStack
    path = tmp_path / "complex.mrc"
    write_stack(path, np.zeros((1, 2, 2), np.float32), 2)
    with open(path, "r+b") as f:  # mode 4: complex 32-bit transform
        f.seek(12)
        f.write(np.int32(4).tobytes())
    with pytest.raises(EttentionError) as e:
        MRCStack(str(path)).load_projections()
    assert e.value.status == _abi.ERR_UNSUPPORTED
    assert "Format of the MRC stack is either unknown or not supported (mode 4)" in str(e.value)
    with pytest.raises(EttentionError) as e:
        MRCStack(str(tmp_path / "missing.mrc"))
    assert "Could not open MRC stack" in str(e.value)


def test_tilt_angle_file(tmp_path):
    from ettention_b200.operators import MRCStack, read_tilt_angles
    t = tmp_path / "a.tlt"
    t.write_text(" -60.5\n-30\n\n  0.25 30\n60.0\n")
    assert read_tilt_angles(str(t)) == [-60.5, -30.0, 0.25, 30.0, 60.0]
    path = tmp_path / "s.mrc"
    write_stack(path, np.zeros((5, 4, 6), np.float32), 2)
    st = MRCStack(str(path), str(t))
    assert st.tilt_angles == [-60.5, -30.0, 0.25, 30.0, 60.0]
    g = st.createScannerGeometry(1)
    from ettention_b200.operators import mrc_base_geometry
    assert np.array_equal(g.projection_matrix(), mrc_base_geometry(6, 4).rotated(-30.0).projection_matrix())
    write_stack(path, np.zeros((4, 4, 6), np.float32), 2)
    with pytest.raises(EttentionError) as e:
        MRCStack(str(path), str(t))
    assert "Number of projections DIFFERS from number of Tilt Angles" in str(e.value)


@pytest.mark.parametrize("orientation", ["xyz", "xzy"])
def test_volume_writer_orders_and_header(tmp_path, orientation):
    from ettention_b200.operators import MRCStack, write_mrc_volume
    rng = np.random.Generator(np.random.PCG64(3))
    vol = rng.normal(size=(6, 5, 7)).astype(np.float32)  # (z, y, x)
    path = tmp_path / "v.mrc"
    write_mrc_volume(str(path), vol, orientation)
    st = MRCStack(str(path))
    back = st.load_projections()
    if orientation == "xyz":
        assert (st.info.nx, st.info.ny, st.info.nz) == (7, 5, 6)
        assert np.array_equal(back, vol)
    else:  # sections = y, rows = z
        assert (st.info.nx, st.info.ny, st.info.nz) == (7, 6, 5)
        assert np.array_equal(back, np.transpose(vol, (1, 0, 2)))
    assert st.info.mode == 2 and st.info.extended_bytes == 0
    assert st.info.dmin == vol.min() and st.info.dmax == vol.max()
    assert st.info.dmean == pytest.approx(float(vol.astype(np.float64).mean()), rel=1e-6)
    with open(path, "rb") as f:
        hdr = f.read(1024)
    assert hdr[208:212] == b"MAP "


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="ETTENTION_REFERENCE (reference checkout) not set")
def test_reference_jason64_stack_and_tilt_file():
    from ettention_b200.operators import MRCStack
    st = MRCStack(os.path.join(REF_DATA, "jason64.ali"), os.path.join(REF_DATA, "jason64.tlt"), logarithmize=True)
    assert (st.info.nx, st.info.ny, st.info.nz, st.info.mode) == (64, 64, 90, 1)
    assert st.info.extended_bytes == 11520
    assert len(st.tilt_angles) == 90 and st.tilt_angles[0] == pytest.approx(-62.78)
    with open(os.path.join(REF_DATA, "jason64.ali"), "rb") as f:
        f.seek(1024 + 11520)
        raw = np.frombuffer(f.read(64 * 64 * 90 * 2), np.int16).reshape(90, 64, 64)
    np.testing.assert_allclose(st.load_projections(), log_transform(raw, 1), rtol=2e-7, atol=1e-7)


def _reference_statistics(v):
    """VolumeStatistics::compute (VolumeStatistics.cpp:17-48) in float32: min from FLT_MAX,
    max from FLT_MIN (the smallest positive normal), NaN skipped, float sum in voxel order
    times 1 / (float)count."""
    f = np.float32
    mn, mx, s = f(np.finfo(np.float32).max), f(np.finfo(np.float32).tiny), f(0.0)
    for x in v.reshape(-1):
        if np.isnan(x):
            continue
        mn = min(mn, x)
        mx = max(mx, x)
        s = f(s + x)
    return mn, mx, f(s * f(f(1.0) / f(v.size)))


def _linear(v, smin, smax, lo, hi):
    """LinearRangeTransformation::transformRange, float32 step by step."""
    f = np.float32
    a = (np.asarray(v, f) - f(smin)).astype(f)
    b = (a / f(f(smax) - f(smin))).astype(f)
    c = (b * f(f(hi) - f(lo))).astype(f)
    return (c + f(lo)).astype(f)


def _mrc_writer_volume():
    """MRCWriterTest's volume (test/src/unit/io/MRCWriterTest.cpp:35-42): 16^3 zeros with
    four voxels set, (z, y, x)."""
    v = np.zeros((16, 16, 16), np.float32)
    v[0, 0, 0], v[0, 0, 15], v[0, 15, 0], v[15, 0, 0] = 1.0, 2.0, 3.0, 4.0
    return v


def _read_mrc(path):
    with open(path, "rb") as fh:
        raw = fh.read()
    hdr = np.frombuffer(raw[:1024], np.uint8)
    nx, ny, nz, mode = np.frombuffer(hdr[:16].tobytes(), np.int32)
    dmin, dmax, dmean = np.frombuffer(hdr[76:88].tobytes(), np.float32)
    dt = {0: np.uint8, 1: np.int16, 2: np.float32, 6: np.uint16}[int(mode)]
    data = np.frombuffer(raw[1024:], dt).reshape(nz, ny, nx)
    return int(mode), (dmin, dmax, dmean), data, raw[208:212]


@pytest.mark.parametrize("vt,mode,lo,hi,dtype", [("unsigned8", 0, 0.0, 255.0, np.uint8),
                                                 ("unsigned16", 6, 0.0, 65535.0, np.uint16),
                                                 ("signed16", 1, -32768.0, 32767.0, np.int16)])
@pytest.mark.parametrize("invert", [False, True])
def test_volume_writer_integer_types_follow_range_transformation(tmp_path, vt, mode, lo, hi, dtype, invert):
    """The MRCWriterTest cases (unsigned 8 / 16, signed 16, inverted): the volume's
    [min, max] mapped linearly onto the type's range (reversed with invert), C-cast, and
    the header's min / max / mean transformed the same way."""
    from ettention_b200.operators import write_mrc_volume
    v = _mrc_writer_volume()
    v[3, 4, 5] = -1.5  # a negative voxel so that the range does not start at zero
    path = tmp_path / "t.mrc"
    write_mrc_volume(str(path), v, "xyz", vt, invert)
    got_mode, hdr, data, tag = _read_mrc(path)
    mn, mx, mean = _reference_statistics(v)
    out_lo, out_hi = (hi, lo) if invert else (lo, hi)
    want = np.trunc(_linear(v, mn, mx, out_lo, out_hi)).astype(dtype)
    assert got_mode == mode and tag == b"MAP "
    assert np.array_equal(data, want)
    assert hdr == tuple(_linear(np.array([mn, mx, mean]), mn, mx, out_lo, out_hi))
    assert data.max() == int(hi) and data.min() == int(lo)


def test_volume_writer_float32_statistics_and_inverted_header(tmp_path):
    """float32 (MRCWriterTest Test_Float32 / Test_Float_32_Inverted): data as is; the
    header carries the reference's statistics -- with invert mapped onto [max, min] while
    the data stay untransformed -- and the XZY order puts y in the sections."""
    from ettention_b200.operators import write_mrc_volume
    v = -np.abs(_mrc_writer_volume()) - 0.25  # all negative: max stays FLT_MIN in the reference
    for invert in (False, True):
        path = tmp_path / f"f{int(invert)}.mrc"
        write_mrc_volume(str(path), v, "xzy", "float32", invert)
        mode, hdr, data, _ = _read_mrc(path)
        mn, mx, mean = _reference_statistics(v)
        assert mode == 2 and np.array_equal(data, np.transpose(v, (1, 0, 2)))
        assert mx == np.finfo(np.float32).tiny
        want = (mn, mx, mean) if not invert else tuple(_linear(np.array([mn, mx, mean]), mn, mx, mx, mn))
        assert hdr == want


def test_volume_writer_rejects_unknown_voxel_type(tmp_path):
    from ettention_b200.operators import EttentionError, write_mrc_volume
    with pytest.raises(EttentionError, match="Unknown file mode"):
        write_mrc_volume(str(tmp_path / "x.mrc"), np.zeros((2, 2, 2), np.float32), "xyz", "float64")
