"""The C++ operator surface (include/ettention_b200.hpp) builds warning-free against
the C ABI and maps onto it on the host: the same projection matrices and traversal
lengths as the Python mirror, the reference's configuration keys and error messages,
and device errors rethrown as GPUException (no device here: status 6)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ettention_b200")


def build_and_run(tmp_path, src, extra=()):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "prog")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), *extra,
           os.path.join(ROOT, "tests", "cpp", src), "-L", LIBDIR, "-lettention_b200", f"-Wl,-rpath,{LIBDIR}",
           "-o", exe]
    if "-lcudart" in extra:
        cmd = cmd[:-2] + ["-L", "/usr/local/cuda/lib64", "-lcudart"] + cmd[-2:]
    subprocess.check_call(cmd)
    return exe


def test_cpp_shim_host_side(tmp_path):
    from ettention_b200.operators import mrc_base_geometry
    exe = build_and_run(tmp_path, "shim_cpu.cpp")
    out = subprocess.run([exe, str(tmp_path / "v.mrc")], capture_output=True, text=True, timeout=120,
                         check=True).stdout
    lines = {l.split()[0] + (" " + l.split()[1] if l.startswith("config") else ""): l.split()
             for l in out.splitlines()}
    g = mrc_base_geometry(96, 80).rotated(30.0)
    m = np.array([float(v) for v in lines["matrix"][1:]], np.float32)
    assert np.array_equal(m, g.projection_matrix())
    t = float(lines["traversal"][1])
    assert t == pytest.approx(g.traversal_length([-48, -40, -20], [48, 40, 20]), rel=1e-7)
    assert lines["config sart"][2:] == ["ok", "1", "5", "0.3", "0", "1"]
    assert lines["config sirt"][2:4] == ["ok", str(0xffffffff)]
    assert lines["config block"][2:] == ["ok", "8", "2", "0.2", "2", "3"]
    assert " ".join(lines["config zero_block"][2:]) == "error 1 Illegal ProjectionBlockSize!"
    assert " ".join(lines["config bad_order"][2:]) == "error 1 Illegal ProjectionSetType!"
    assert lines["config missing"][2:4] == ["error", "1"]
    assert lines["mrc"][1:] == ["ok", "0", "23"]
    assert lines["mrc_missing"][1:] == ["error", "1"]
    assert lines["stack"][1:] == ["2", "6", "5", "-30", "45.5", "1.75", "-1.75"]
    assert lines["tiff"][1:] == ["6", "5", "7.25"]
    assert lines["xml"][1:] == ["sirt", "4", "0.5", "/sub/dir"]
    from oracle import oracle as O
    blob = O.blob_ray_integration_samples(O.BlobParameters(), 4)
    assert [float(v) for v in lines["blob"][1:]] == pytest.approx([blob[0], blob[1], blob[3]], abs=1e-6)
    import torch
    if torch.cuda.is_available():
        assert lines["framework"][1] == "ok"
    else:
        assert lines["framework"][1:3] == ["gpu_error", "6"]
