"""SyntheticReconstruction.cpp:66-172 through the reference's front door, on the GPU.

The data set is made the way the reference made synthetic_3_parallel: the ground
truth (committed fixture) forward projected at -90..89 degrees with the
ProjectionTestBase geometry (here by the CUDA forward projector; five projections
are checked against the reference's own files), written as 32-bit float TIFFs with a
metadata.xml.  Parameter files with the settings of the reference's sart.xml,
sirt.xml and blockIterative.xml (4 sub-volumes; projection order left at its
default) are run by reconstruct_from_config: XML parameters, the directory
datasource, the CUDA reconstruction and the XZY MRC writer.  The written volume must
be within the reference's own bounds of the ground truth: max slice RMS <= 0.7 /
0.7 / 0.2 over the file's sections."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONFIGS = {
    "sart": ('<algorithm value="sart"><numberOfIterations value="2"/><useLongObjectCompensation value="false"/>'
             '<lambda value="0.1"/></algorithm><backProjection><samples value="9"/></backProjection>'
             '<forwardProjection><samples value="4"/></forwardProjection>', 0.7),
    "sirt": ('<algorithm value="sirt"><numberOfIterations value="25"/><useLongObjectCompensation value="false"/>'
             '<lambda value="1.0"/></algorithm><backProjection><samples value="1"/></backProjection>'
             '<forwardProjection><samples value="1"/></forwardProjection>', 0.7),
    "blockIterative": ('<algorithm value="blockIterative"><blockSize value="10"/><numberOfIterations value="10"/>'
                       '<lambda value="1.0"/></algorithm>', 0.2),
}


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    from oracle import oracle as O
    from ettention_b200.operators import (Context, ForwardProjectionOperator, GPUMappedVolume,
                                          ImageStackDirectoryDatasource, write_mrc_volume, write_tiff)
    from tests.helpers import golden, product_geometry, xzy_to_zyx
    import torch
    d = tmp_path_factory.mktemp("synthetic_3_parallel")
    syn = golden("synth")
    truth = xzy_to_zyx(syn["ground_truth"])  # the fixture is the XZY file; the volume is (z, y, x)
    base = product_geometry(O.projection_test_geometry())
    angles = list(range(-90, 90))
    ctx = Context(0)
    vol = GPUMappedVolume(ctx, (64, 64, 64))
    vol.upload(truth)
    fp = ForwardProjectionOperator(vol, 1)
    names = []
    for a in angles:
        p = torch.zeros((256, 256), dtype=torch.float32, device="cuda")
        fp.setScannerGeometry(base.rotated(float(a)))
        fp.SetOutput(p, torch.zeros_like(p))
        fp.Execute(0)
        ctx.synchronize()
        img = p.cpu().numpy()
        if a in [int(x) for x in syn["angles"]]:
            assert O.images_equal(img, syn[f"projection_{a}"])
        names.append(f"projection{a}.tif")
        write_tiff(str(d / names[-1]), img)
    vol.close()
    ctx.close()
    ImageStackDirectoryDatasource.writeMetaDataFile(str(d / "metadata.xml"), [float(a) for a in angles], names, base,
                                                    (64, 64, 64))
    write_mrc_volume(str(d / "ground_truth.mrc"), truth)
    return d


@pytest.mark.parametrize("name", list(CONFIGS))
def test_reference_parameter_files_reconstruct_within_bounds(dataset, name):
    from oracle import oracle as O
    from ettention_b200.operators import MRCStack, XMLParameterSource, reconstruct_from_config
    body, limit = CONFIGS[name]
    xml = dataset / f"{name}.xml"
    xml.write_text('<?xml version="1.0"?>\n<hardware><subVolumeCount value="4"/></hardware>\n' + body +
                   '<input><projections value="."/></input>'
                   f'<output><filename value="out\\generated_{name}.mrc"/>'
                   '<options><voxelType value="float32"/></options></output>'
                   '<volume><dimension value="64 64 64"/><initValue value="0.0"/></volume>')
    (dataset / "out").mkdir(exist_ok=True)
    v = reconstruct_from_config(XMLParameterSource(str(xml)))
    written = MRCStack(str(dataset / "out" / f"generated_{name}.mrc")).load_projections()
    truth = MRCStack(str(dataset / "ground_truth.mrc")).load_projections()
    assert written.shape == (64, 64, 64)
    assert np.array_equal(written, np.transpose(v, (1, 0, 2)))  # XZY: sections are y
    rms = O.max_slice_rms(written, truth)
    assert rms <= limit, rms


@pytest.mark.parametrize("vt,invert,dtype", [("unsigned16", "true", np.uint16), ("unsigned8", "false", np.uint8)])
def test_parameter_file_output_voxel_type_and_invert(dataset, vt, invert, dtype):
    """output.options.voxelType / invert through the front door: the written file is the
    reconstruction mapped onto the type's range (reversed with invert) in XZY order."""
    from ettention_b200.operators import XMLParameterSource, reconstruct_from_config
    body, _ = CONFIGS["sart"]
    xml = dataset / f"out_{vt}.xml"
    xml.write_text('<?xml version="1.0"?>\n' + body + '<input><projections value="."/></input>'
                   f'<output><filename value="out/typed_{vt}.mrc"/>'
                   f'<options><voxelType value="{vt}"/><invert value="{invert}"/></options></output>'
                   '<volume><dimension value="64 64 64"/><initValue value="0.0"/></volume>')
    (dataset / "out").mkdir(exist_ok=True)
    v = reconstruct_from_config(XMLParameterSource(str(xml)))
    with open(dataset / "out" / f"typed_{vt}.mrc", "rb") as fh:
        raw = fh.read()
    mode = int(np.frombuffer(raw[12:16], np.int32)[0])
    data = np.frombuffer(raw[1024:], dtype).reshape(64, 64, 64)
    assert mode == {"unsigned16": 6, "unsigned8": 0}[vt]
    top = int(np.iinfo(dtype).max)
    lo_voxel, hi_voxel = np.unravel_index(np.argmin(v), v.shape), np.unravel_index(np.argmax(v), v.shape)
    xzy = lambda i: (i[1], i[0], i[2])  # noqa: E731 (z, y, x) index -> file (y, z, x)
    if invert == "true":
        assert data[xzy(lo_voxel)] == top and data[xzy(hi_voxel)] == 0
    else:
        assert data[xzy(lo_voxel)] == 0 and data[xzy(hi_voxel)] == top
