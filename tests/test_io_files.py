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
