"""Directory image stacks (metadata.xml + TIFF projections) and XML parameter files, the
reference's other front door (LR/io/datasource/ImageStackDirectoryDatasource.cpp,
LR/io/deserializer/ImageDeserializer.cpp, LR/setup/parametersource/XMLParameterSource.cpp).

The TIFF decoder is checked against Pillow's libtiff (an independent decoder and
encoder) over the compressions, predictors, sample types and layouts it supports,
and, where the reference checkout is present, over the 180 LZW projections of its
synthetic_3_parallel data set.  Host-only: no GPU."""
import os
import struct

import numpy as np
import pytest

from tests.helpers import reference_path

REF_SYNTH = reference_path("ettention", "test", "data", "synthetic_3_parallel")


def _rand(shape, seed=0):
    return np.random.default_rng(seed).standard_normal(shape).astype(np.float32)


@pytest.mark.parametrize("compression", ["raw", "tiff_lzw", "tiff_adobe_deflate", "packbits"])
@pytest.mark.parametrize("predictor", [1, 3])
def test_float_tiff_matches_libtiff(tmp_path, compression, predictor):
    from PIL import Image
    from ettention_b200.operators import read_tiff
    if predictor == 3 and compression in ("raw", "packbits"):
        pytest.skip("predictors apply to LZW and Deflate")
    a = _rand((37, 53), 1)
    a[0, 0], a[5, 7] = np.inf, -0.0
    path = str(tmp_path / "f.tif")
    info = {317: predictor} if predictor != 1 else {}
    Image.fromarray(a, "F").save(path, compression=compression, tiffinfo={278: 5, **info})
    assert np.array_equal(np.array(Image.open(path), np.float32), a)
    got = read_tiff(path)
    assert got.shape == a.shape
    assert np.array_equal(got.view(np.uint32), a.view(np.uint32))


@pytest.mark.parametrize("dtype,compression", [(np.uint8, "tiff_lzw"), (np.uint8, "tiff_adobe_deflate"),
                                               (np.uint16, "tiff_lzw"), (np.uint16, "raw")])
def test_integer_tiff_is_normalised_like_freeimage(tmp_path, dtype, compression):
    """8-bit grey / 255, 16-bit grey / 65535 (FreeImage's conversion to float)."""
    from PIL import Image
    from ettention_b200.operators import read_tiff
    hi = np.iinfo(dtype).max
    a = np.random.default_rng(2).integers(0, hi + 1, (19, 23)).astype(dtype)
    a[0, 0], a[1, 1] = 0, hi
    path = str(tmp_path / "i.tif")
    Image.fromarray(a).save(path, compression=compression, tiffinfo={317: 2} if compression != "raw" else {})
    assert np.array_equal(read_tiff(path), a.astype(np.float32) / np.float32(hi))


def _write_tiff_by_hand(path, a, big_endian=False, tile=None):
    """An uncompressed float32 TIFF written field by field: big-endian and/or tiled."""
    e = ">" if big_endian else "<"
    H, W = a.shape
    if tile:
        th, tw = tile
        blocks = []
        for ty in range(0, H, th):
            for tx in range(0, W, tw):
                t = np.zeros((th, tw), np.float32)
                part = a[ty:ty + th, tx:tx + tw]
                t[:part.shape[0], :part.shape[1]] = part
                blocks.append(t.astype(e + "f4").tobytes())
    else:
        blocks = [a.astype(e + "f4").tobytes()]
    n = len(blocks)
    entries = [(256, 4, 1, W), (257, 4, 1, H), (258, 3, 1, 32), (259, 3, 1, 1), (262, 3, 1, 1), (277, 3, 1, 1),
               (339, 3, 1, 3)]
    data_at = 1024 + 8 * n
    offs = []
    pos = data_at
    for b in blocks:
        offs.append(pos)
        pos += len(b)
    if tile:
        entries += [(322, 4, 1, tile[1]), (323, 4, 1, tile[0]), (324, 4, n, 1024), (325, 4, n, 1024 + 4 * n)]
    else:
        entries += [(273, 4, 1, offs[0]), (278, 4, 1, H), (279, 4, 1, len(blocks[0]))]
    entries.sort()
    out = bytearray(b"MM" if big_endian else b"II")
    out += struct.pack(e + "HI", 42, 8)
    out += struct.pack(e + "H", len(entries))
    for tag, typ, cnt, val in entries:
        out += struct.pack(e + "HHI", tag, typ, cnt)
        out += struct.pack(e + "HH", val, 0) if typ == 3 and cnt == 1 else struct.pack(e + "I", val)
    out += struct.pack(e + "I", 0)
    out += b"\0" * (1024 - len(out))
    out += b"".join(struct.pack(e + "I", o) for o in offs) + b"".join(struct.pack(e + "I", len(b)) for b in blocks)
    assert len(out) == data_at
    out += b"".join(blocks)
    with open(path, "wb") as f:
        f.write(bytes(out))


@pytest.mark.parametrize("big_endian,tile", [(True, None), (False, (16, 16)), (True, (16, 32))])
def test_byte_order_and_tiles(tmp_path, big_endian, tile):
    from PIL import Image
    from ettention_b200.operators import read_tiff
    a = _rand((37, 53), 3)
    path = str(tmp_path / "h.tif")
    _write_tiff_by_hand(path, a, big_endian, tile)
    assert np.array_equal(np.array(Image.open(path), np.float32), a)  # the file itself is valid
    assert np.array_equal(read_tiff(path), a)


def test_tiff_writer_round_trip_and_pages(tmp_path):
    from PIL import Image
    from ettention_b200.operators import read_tiff, tiff_page_count, write_tiff
    a = _rand((31, 47), 4)
    path = str(tmp_path / "w.tif")
    write_tiff(path, a)
    assert np.array_equal(np.array(Image.open(path), np.float32), a)  # readable by libtiff
    assert np.array_equal(read_tiff(path), a)
    multi = str(tmp_path / "m.tif")
    Image.fromarray(a, "F").save(multi, save_all=True, compression="tiff_lzw",
                                 append_images=[Image.fromarray(a * 2, "F"), Image.fromarray(a * 3, "F")])
    assert tiff_page_count(multi) == 3
    for k in range(3):
        assert np.array_equal(read_tiff(multi, k), a * (k + 1))


def test_tiff_errors(tmp_path):
    from PIL import Image
    from ettention_b200 import _abi
    from ettention_b200.operators import EttentionError, read_tiff
    rgb = str(tmp_path / "rgb.tif")
    Image.fromarray(np.zeros((4, 4, 3), np.uint8), "RGB").save(rgb)
    with pytest.raises(EttentionError, match="grey images") as e:
        read_tiff(rgb)
    assert e.value.status == _abi.ERR_UNSUPPORTED
    i32 = str(tmp_path / "i32.tif")
    Image.fromarray(np.zeros((4, 4), np.int32), "I").save(i32)
    with pytest.raises(EttentionError, match="cannot be converted to float"):
        read_tiff(i32)
    with pytest.raises(EttentionError, match="unable to load image"):
        read_tiff(str(tmp_path / "missing.tif"))
    junk = tmp_path / "junk.tif"
    junk.write_bytes(b"not a tiff at all")
    with pytest.raises(EttentionError, match="not a TIFF"):
        read_tiff(str(junk))
    with pytest.raises(EttentionError, match="index out of bound"):
        read_tiff(rgb, 3)
    # a strip that claims bytes past the end of the file
    a = _rand((8, 8), 5)
    ok = str(tmp_path / "ok.tif")
    _write_tiff_by_hand(ok, a)
    cut = tmp_path / "cut.tif"
    cut.write_bytes(open(ok, "rb").read()[:-40])
    with pytest.raises(EttentionError, match="outside the file"):
        read_tiff(str(cut))


# ----------------------------------------------------------------------------- directory stacks
def _make_stack(tmp_path, angles, logscale=(), stack_pages=None):
    from ettention_b200.operators import ImageStackDirectoryDatasource, ScannerGeometry, write_tiff
    base = ScannerGeometry([-8.0, -6.0, -32.0], [-8.0, -6.0, 32.0], [0.5, 0.0, 0.0], [0.0, 0.5, 0.0], 32, 24)
    names, imgs = [], []
    for k, a in enumerate(angles):
        img = _rand((24, 32), 10 + k)
        name = f"projection{a:g}.tif"
        write_tiff(str(tmp_path / name), img)
        names.append(name)
        imgs.append(img)
    ImageStackDirectoryDatasource.writeMetaDataFile(str(tmp_path / "metadata.xml"), angles, names, base, (16, 16, 8))
    return base, names, imgs


def test_directory_stack_round_trip(tmp_path):
    from ettention_b200.operators import ImageStackDirectoryDatasource, open_image_stack
    angles = [-60.0, -12.5, 0.0, 33.25, 60.0]
    base, names, imgs = _make_stack(tmp_path, angles)
    ds = open_image_stack(str(tmp_path))
    assert isinstance(ds, ImageStackDirectoryDatasource)
    assert ds.getNumberOfProjections() == 5 and ds.getResolution() == (32, 24)
    assert ds.tilt_angles == angles
    assert np.allclose(ds.base_geometry.source, base.source) and np.allclose(ds.base_geometry.hpitch, base.hpitch)
    assert ds.base_geometry.width == 32 and ds.base_geometry.height == 24 and not ds.base_geometry.perspective
    data = ds.load_projections()
    assert np.array_equal(data, np.stack(imgs))
    assert np.array_equal(ds.getProjectionImage(3), imgs[3])
    assert np.array_equal(ds.load_projections(1, 2), np.stack(imgs[1:3]))
    g = ds.createScannerGeometry(1, 2.0)
    r = base.rotated(-12.5, 2.0)
    assert np.allclose(g.source, r.source) and np.allclose(g.vpitch, r.vpitch)
    ds.close()


def test_metadata_logscale_stacks_and_repeated_angles(tmp_path):
    """<logscale/> exponentiates (Image::convertToLinearScale); a <projectionstack> gives one
    projection per page at one tilt angle; repeated angles are numbered after the
    angle's first appearance (the reference's (angle, repeat) hyper-stack index)."""
    from PIL import Image
    from ettention_b200.operators import ImageStackDirectoryDatasource, write_tiff
    a0, a1, a2 = _rand((6, 5), 1), _rand((6, 5), 2), _rand((6, 5), 3)
    write_tiff(str(tmp_path / "a0.tif"), a0)
    write_tiff(str(tmp_path / "a1.tif"), a1)
    Image.fromarray(a2, "F").save(str(tmp_path / "pages.tif"), save_all=True, compression="tiff_lzw",
                                  append_images=[Image.fromarray(a2 + 1, "F")])
    (tmp_path / "metadata.xml").write_text("""<?xml version="1.0"?>
<!-- a comment -->
<geometry>
  <sourcePosition value="0 0 -10"/><detectorPosition value=" 0 0 10 "/>
  <horizontalPitch value='1 0 0'/><verticalPitch value="0 1 0"/>
</geometry>
<projection><image filename="a0.tif"/><tiltAngle value="5"/></projection>
<projectionstack><image filename="pages.tif"/><tiltAngle value="-5"/></projectionstack>
<projection><image filename="a1.tif"/><tiltAngle value="5"/><logscale/></projection>
""")
    ds = ImageStackDirectoryDatasource(str(tmp_path))
    # angle 5 first appeared first: (0,0)=a0, (0,1)=a1 (logscale), then (1,0), (1,1) = pages
    assert ds.tilt_angles == [5.0, 5.0, -5.0, -5.0]
    d = ds.load_projections()
    assert np.array_equal(d[0], a0)
    assert np.allclose(d[1], np.exp(a1.astype(np.float64)), rtol=2e-7, atol=0)  # libm expf: within 1 ulp
    assert np.array_equal(d[2], a2) and np.array_equal(d[3], a2 + 1)


def test_metadata_errors(tmp_path):
    from ettention_b200.operators import EttentionError, ImageStackDirectoryDatasource, open_image_stack, write_tiff
    with pytest.raises(EttentionError, match="Unable to open image stack"):
        open_image_stack(str(tmp_path))
    write_tiff(str(tmp_path / "a.tif"), _rand((4, 4)))
    geo = ('<geometry><sourcePosition value="0 0 -1"/><detectorPosition value="0 0 1"/>'
           '<horizontalPitch value="1 0 0"/><verticalPitch value="0 1 0"/></geometry>')
    cases = [
        ('<projection><image filename="a.tif"/><tiltAngle value="1"/></projection>', "No such node \\(geometry\\)"),
        (geo + '<projection><image filename="a.tif"/></projection>', "No such node \\(tiltAngle\\)"),
        (geo + '<projection><image filename="a.tif"/><tiltAngle value="x"/></projection>', "conversion"),
        (geo + '<projection><image filename="b.tif"/><tiltAngle value="1"/></projection>', "unable to load image"),
        (geo + '<projection><image filename="a.tif"/><tiltAngle value="1"/></projectio>', "mismatched end tag"),
        (geo, "lists no projections"),
        (geo.replace('"1 0 0"', '"1 0"') + '<projection><image filename="a.tif"/><tiltAngle value="1"/></projection>',
         "conversion of data to a vector"),
    ]
    for text, msg in cases:
        (tmp_path / "metadata.xml").write_text(text)
        with pytest.raises(EttentionError, match=msg):
            ImageStackDirectoryDatasource(str(tmp_path))
    # an image of another size than the first one is reported when loading
    write_tiff(str(tmp_path / "big.tif"), _rand((5, 4)))
    (tmp_path / "metadata.xml").write_text(geo + '<projection><image filename="a.tif"/><tiltAngle value="1"/>'
                                           '</projection><projection><image filename="big.tif"/>'
                                           '<tiltAngle value="2"/></projection>')
    ds = ImageStackDirectoryDatasource(str(tmp_path))
    with pytest.raises(EttentionError, match="the stack's projections are 4 x 4"):
        ds.load_projections()


def test_xml_parameter_source(tmp_path):
    from ettention_b200.operators import AlgebraicParameterSet, XMLParameterSource
    (tmp_path / "cfg").mkdir()
    cfg = tmp_path / "cfg" / "run.xml"
    cfg.write_text("""<?xml version="1.0"?>
<hardware><subVolumeCount value="4" /></hardware>
<algorithm value="blockIterative" >
  <blockSize value="10" /><!-- ignored --><numberOfIterations value="3" /><lambda value="0.5" />
</algorithm>
<algorithm value="sirt"><blockSize value="99"/></algorithm>
<input><projections value="..\\data"/><tiltAngles value="/abs/t.tlt"/></input>
<output><filename value="out/vol.mrc"/><options><orientation value="xyz_order"/></options></output>
<volume><dimension value="64 64 32"/><origin value="1 &amp; 2"/></volume>
""")
    src = XMLParameterSource(str(cfg))
    assert src.getStringParameter("algorithm") == "blockIterative"  # the first element wins
    assert src.getStringParameter("algorithm.blockSize") == "10"
    assert src.getStringParameter("volume.origin") == "1 & 2"
    assert src.getStringParameter("output.options.orientation") == "xyz_order"
    c = src.config()
    assert c["input.projections"] == str(tmp_path / "data")
    assert c["input.tiltAngles"] == "/abs/t.tlt"
    assert c["output.filename"] == str(tmp_path / "cfg" / "out" / "vol.mrc")
    assert not src.parameterExists("debug.writeProjections")
    p = AlgebraicParameterSet.from_config({k: v for k, v in c.items() if k != "volume.origin"})
    assert (p.block_size, p.iterations, p.lam, p.subvolume_count, list(p.resolution)) == (10, 3, 0.5, 4, [64, 64, 32])


def test_init_and_mask_volumes(tmp_path):
    """volume.initFile in each coordinate order; the mask file is read in file order."""
    from ettention_b200.operators import EttentionError, load_init_volume, load_mask_volume, write_mrc_volume
    v = _rand((5, 6, 7), 9)  # (z, y, x): X=7, Y=6, Z=5
    write_mrc_volume(str(tmp_path / "xzy.mrc"), v, "xzy")
    write_mrc_volume(str(tmp_path / "xyz.mrc"), v, "xyz")
    assert np.array_equal(load_init_volume(str(tmp_path / "xzy.mrc"), "xzy_order", (7, 6, 5)), v)
    assert np.array_equal(load_init_volume(str(tmp_path / "xyz.mrc"), "xyz_order", (7, 6, 5)), v)
    # file coordinates (x, y, z) of an XYZ file read as ZYX: working (x, y, z) = file (z, y, x)
    w = load_init_volume(str(tmp_path / "xyz.mrc"), "zyx_order", (5, 6, 7))
    assert np.array_equal(w, np.transpose(v, (2, 1, 0)))
    with pytest.raises(EttentionError, match="does not match resolution"):
        load_init_volume(str(tmp_path / "xzy.mrc"), "xyz_order", (7, 6, 5))
    with pytest.raises(EttentionError, match="Unknown CoordinateOrder"):
        load_init_volume(str(tmp_path / "xzy.mrc"), "abc_order", (7, 6, 5))
    m = np.array([[[0.0, 1.0, 200.7, 300.0, -3.0, 254.99, 7.0]] * 6] * 5, np.float32)
    write_mrc_volume(str(tmp_path / "mask.mrc"), m, "xyz")
    got = load_mask_volume(str(tmp_path / "mask.mrc"), (7, 6, 5))
    assert got.dtype == np.uint8 and list(got[0, 0]) == [0, 1, 200, 255, 0, 254, 7]


# ----------------------------------------------------------------------------- the reference's data set
@pytest.mark.skipif(not os.path.isdir(REF_SYNTH), reason="ETTENTION_REFERENCE (reference checkout) not set")
def test_reference_synthetic_directory_stack():
    """synthetic_3_parallel: 180 LZW float projections, metadata.xml, sart/sirt/blockIterative
    parameter files, read through the native reader."""
    from PIL import Image
    from oracle import oracle as O
    from ettention_b200.operators import AlgebraicParameterSet, XMLParameterSource, open_image_stack
    from tests.helpers import golden
    cfg = XMLParameterSource(os.path.join(REF_SYNTH, "blockIterative.xml")).config()
    assert cfg["input.projections"] == REF_SYNTH
    p = AlgebraicParameterSet.from_config(cfg)
    assert (p.algorithm, p.block_size, p.iterations, p.lam, p.subvolume_count) == ("blockIterative", 10, 10, 1.0, 4)
    ds = open_image_stack(cfg["input.projections"])
    assert ds.tilt_angles == [float(a) for a in range(-90, 90)]
    base = O.projection_test_geometry()
    for name in ("source", "detector", "hpitch", "vpitch"):
        assert np.array_equal(np.float32(getattr(ds.base_geometry, name)), np.float32(getattr(base, name)))
    data = ds.load_projections()
    for k, a in enumerate(ds.tilt_angles):
        ref = np.array(Image.open(os.path.join(REF_SYNTH, f"projection{int(a)}.tif")), np.float32)
        assert np.array_equal(data[k], ref), a
    syn = golden("synth")
    for a in syn["angles"]:
        assert np.array_equal(data[ds.tilt_angles.index(float(a))], syn[f"projection_{int(a)}"])
    for name, algo, iters, lam, fs, bs in (("sart", "sart", 2, 0.1, 4, 9), ("sirt", "sirt", 25, 1.0, 1, 1)):
        q = AlgebraicParameterSet.from_config(XMLParameterSource(os.path.join(REF_SYNTH, f"{name}.xml")).config())
        assert (q.algorithm, q.iterations, q.lam, q.fp_samples, q.bp_samples) == (algo, iters, lam, fs, bs)
