"""The host driver's VTI writer on the CPU: a small C++ harness links
host/complab_io.cpp, writes known arrays, and the file is read back here as
a VTK reader would (XML ImageData, inline base64 with a UInt64 byte count,
x fastest, the interior planes x = 1..nx-2 only), and the reference's file
names (7-digit steps)."""
import base64
import os
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from test_driver_config import DRIVER, driver_available

HOST = os.path.join(os.path.dirname(DRIVER), "host")

HARNESS = r"""
#include "complab_io.h"
#include <cstdio>
int main(int argc, char** argv) {
    const int nx = 5, ny = 3, nz = 2;
    const size_t N = (size_t)nx * ny * nz;
    clhost::VtiArray a{"Density", 1, true, std::vector<double>(N)};
    clhost::VtiArray v{"velocity", 3, false, std::vector<double>(3 * N)};
    for (size_t n = 0; n < N; ++n) {
        a.data[n] = 0.5 + (double)n;
        for (int c = 0; c < 3; ++c) v.data[c * N + n] = 1000.0 * c + (double)n;
    }
    std::string err;
    const std::string path = std::string(argv[1]) + "/" + clhost::vti_name("A_", 200);
    if (!clhost::write_vti(path, nx, ny, nz, {a, v}, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 1; }
    std::printf("%s\n", path.c_str());
    return 0;
}
"""


def decode(da):
    raw = base64.b64decode(da.text.strip())
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    dt = np.float64 if da.get("type") == "Float64" else np.float32
    return np.frombuffer(raw[8:8 + n], dt)


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
def test_vti_layout(tmp_path):
    src = tmp_path / "h.cpp"
    src.write_text(HARNESS)
    exe = str(tmp_path / "h")
    lib_dir = os.path.dirname(DRIVER)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, str(src), os.path.join(HOST, "complab_io.cpp"),
                        os.path.join(HOST, "complab_xml.cpp"), "-I" + HOST, "-L" + lib_dir, "-lcomplab_gpu",
                        "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    path = r.stdout.strip()
    assert os.path.basename(path) == "A_0000200.vti"
    root = ET.parse(path).getroot()
    assert root.get("type") == "ImageData" and root.get("header_type") == "UInt64"
    img = root.find("ImageData")
    assert img.get("WholeExtent") == "0 2 0 2 0 1"          # nx - 2 = 3 interior planes
    arrays = {da.get("Name"): da for da in img.iter("DataArray")}
    nx, ny, nz = 5, 3, 2
    n = np.arange(nx * ny * nz).reshape(nx, ny, nz)
    # VTK point order: x fastest, then y, then z, over x = 1..nx-2
    want = (0.5 + n[1:-1]).transpose(2, 1, 0).reshape(-1)
    np.testing.assert_array_equal(decode(arrays["Density"]), want)
    vel = decode(arrays["velocity"]).reshape(-1, 3)
    assert arrays["velocity"].get("NumberOfComponents") == "3"
    for c in range(3):
        np.testing.assert_array_equal(vel[:, c], (1000.0 * c + n[1:-1]).transpose(2, 1, 0).reshape(-1))
