"""The integration of INTEGRATION.md section 1, built: the reference's own
KDevice wrapper (Interface/KDevice.cpp, compiled unchanged against
include/kdevice/Device/DeviceInterface.h) and project reader
(Input/KSimulationData.cpp), linked with a headless driver against
libblaze_b200.so (oracle/Makefile, target _ref/kdevice_headless; built when
the reference tree is present).

CPU: the binary takes the step interface from the library, by the C names
of DeviceInterface.h.  GPU: it runs the reference's Projects/2.Silo world
SPH_90 (1,950 spheres, the golden fixture's structs and state) for 10 steps
through KDevice and returns the reference kernels' state bit for bit."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import bindings
from conftest import Golden

BIN = os.path.join(os.path.dirname(bindings.REF_SO), "kdevice_headless")
need_bin = pytest.mark.skipif(not os.path.isfile(BIN), reason="oracle/_ref/kdevice_headless not built")

STEP_INTERFACE = ["Device_Set_SimulationData", "Device_Set_System_State", "Device_DEM_UpdateSim",
                  "Device_Get_System_State", "drum_rotation", "Device_Clean"]


@need_bin
def test_kdevice_links_the_library_by_c_names():
    out = subprocess.run(["nm", "-D", "--undefined-only", BIN], capture_output=True, text=True,
                         check=True).stdout.split()
    for name in STEP_INTERFACE:
        assert name in out, name
    libs = subprocess.run(["ldd", BIN], capture_output=True, text=True).stdout
    assert "libblaze_b200.so" in libs


def write_input(path, g):
    z = g.z
    st = g.init()
    n = len(st["pos"])
    sizes = [len(z["sim_info"]), len(z["wobj"]) // 8, len(z["pobj"]) // 8, len(z["dobj"]) // 32]
    head = np.array([0x4B444556, n, g.n_w, g.n_p, g.n_d, int(g.cyl_rot)] + sizes, np.int32)
    with open(path, "wb") as fh:
        for a in (head, z["sim_info"], z["wobj"], z["pobj"], z["dobj"]):
            fh.write(np.ascontiguousarray(a).tobytes())
        for key, dt in (("pos", np.float32), ("vel", np.float32), ("avel", np.float32),
                        ("type", np.uint32), ("pid", np.int32)):
            fh.write(np.ascontiguousarray(st[key], dt).tobytes())
    return n


@pytest.mark.gpu
@need_bin
def test_kdevice_steps_the_reference_silo():
    g = Golden("silo_sph90")
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        n = write_input(src, g)
        rc = subprocess.run([BIN, src, dst, "10"], capture_output=True, text=True)
        assert rc.returncode == 0, (rc.returncode, rc.stderr)
        raw = open(dst, "rb").read()
    f = np.frombuffer(raw, np.float32, count=9 * n).reshape(3, n, 3)
    typ = np.frombuffer(raw, np.uint32, count=n, offset=36 * n)
    pid = np.frombuffer(raw, np.int32, count=n, offset=40 * n)
    ref = g.at(10)
    np.testing.assert_array_equal(f[0], ref["pos"])
    np.testing.assert_array_equal(f[1], ref["vel"])
    np.testing.assert_array_equal(f[2], ref["avel"])
    np.testing.assert_array_equal(typ, ref["type"])
    np.testing.assert_array_equal(pid, ref["pid"])
