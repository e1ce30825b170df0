"""The initial lattice Device_Set_SimulationData lays out for a world that
reads no state file (DeviceInterface.cu:192-707, main.cpp:534-541), on the
reference's own Spheres_128cm box (tests/golden/box_grid.npz: 32,768
spheres on a 32^3 default grid).

Bar: positions, velocities, types and P_IDs equal to a float32 restatement
of the reference's lattice loops bit for bit (default grid; random grid
with glibc rand() from its unseeded start); 20 steps later the state equals
oracle A's started from the same lattice, bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest

import bindings
from blaze import device
from blaze import types as T

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LIBC = ctypes.CDLL("libc.so.6")
RAND_MAX = 2147483647


class Grid:
    def __init__(self):
        z = np.load(os.path.join(HERE, "golden", "box_grid.npz"))
        self.n_w, self.n_p, self.n_d = int(z["n_w"]), int(z["n_p"]), int(z["n_d"])
        self.wobj = (T.WOBJ * 8).from_buffer_copy(z["wobj"].tobytes())
        self.pobj = (T.POBJ * 8).from_buffer_copy(z["pobj"].tobytes())
        self.dobj = (T.DOBJ * 32).from_buffer_copy(z["dobj"].tobytes())
        self.sim_info = T.SimulationInfo.from_buffer_copy(z["sim_info"].tobytes())
        self.init = T.InitConfig.from_buffer_copy(z["init"].tobytes())
        self.per = (ctypes.c_int * 8)(*[int(v) for v in z["per_object"]])
        self.sim_info.Num_ParticlesPerObject = ctypes.cast(self.per, ctypes.POINTER(ctypes.c_int))
        self.n = self.sim_info.Num_Particles


def axis(start, size, space, count):
    out = np.zeros(count, np.float32)
    v = np.float32(start)
    for k in range(count):
        out[k] = v
        v = np.float32(np.float32(v + np.float32(size)) + np.float32(space))
    return out


def restated(g, random=False):
    c = g.init
    NX, NY, NZ = c.num.x, c.num.y, c.num.z
    xs = axis(c.start.x, c.p_size[0].x, c.space.x, NX)
    ys = axis(c.start.y, c.p_size[0].y, c.space.y, NY)
    zs = axis(c.start.z, c.p_size[0].z, c.space.z, NZ)
    Y, Z, X = np.meshgrid(ys, zs, xs, indexing="ij")      # x fastest, then z, then y
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)[:g.n].astype(np.float32)
    per = [g.per[i] for i in range(g.n_p)]
    if not random:
        typ = np.repeat(np.arange(g.n_p), per).astype(np.uint32)
        pid = np.arange(g.n, dtype=np.int32)
    else:
        typ = np.zeros(g.n, np.uint32)
        pid = np.arange(g.n, dtype=np.int32)
        count, sel = [0] * g.n_p, -1
        for k in range(g.n):
            sel = sel + 1 if sel + 1 < g.n_p else 0
            pty = sel
            if count[pty] >= per[pty]:
                pty = next(i for i in range(g.n_p) if count[i] <= per[i] - 1)
            count[pty] += 1
            typ[k] = pty
        for _ in range(g.n):
            a = LIBC.rand() % (g.n - 1)
            b = LIBC.rand() % (g.n - 1)
            typ[a], typ[b] = typ[b], typ[a]
            pid[a], pid[b] = pid[b], pid[a]
    v0 = c.velocity[0]
    vel = np.tile(np.array([v0.x, v0.y, v0.z], np.float32), (g.n, 1))
    return dict(pos=pos, vel=vel, avel=np.zeros((g.n, 3), np.float32), type=typ, pid=pid)


def device_state(g, init):
    kd = device.KDevice(g.wobj, g.pobj, g.dobj, g.n_w, g.n_p, g.n_d, g.sim_info, init)
    out = {k: np.zeros((g.n, 3), np.float32) for k in ("pos", "vel", "avel", "acc")}
    out["type"] = np.zeros(g.n, np.uint32)
    out["pid"] = np.zeros(g.n, np.int32)
    assert kd.IDevice_Get_System_State(out["pos"], None, out["vel"], out["avel"], out["acc"],
                                       out["type"], out["pid"]) == 0
    return kd, out


def test_default_grid_and_trajectory():
    g = Grid()
    kd, got = device_state(g, g.init)
    ref = restated(g)
    for key in ("pos", "vel", "avel", "type", "pid"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)
    if bindings.ref_available():
        R = bindings.RefHost()
        R.init(g.sim_info, g.wobj, g.n_w, g.pobj, g.n_p, g.dobj, g.n_d, threads=8, capture=False)
        R.set_state(ref["pos"], ref["vel"], ref["avel"], ref["type"], ref["pid"])
        assert R.step(20) == 0
        for _ in range(20):
            kd.IDevice_DEM_UpdateSim()
        _, after = None, {k: np.zeros((g.n, 3), np.float32) for k in ("pos", "vel", "avel", "acc")}
        after["type"] = np.zeros(g.n, np.uint32)
        after["pid"] = np.zeros(g.n, np.int32)
        kd.IDevice_Get_System_State(after["pos"], None, after["vel"], after["avel"], after["acc"],
                                    after["type"], after["pid"])
        b = R.state()
        for key in ("pos", "vel", "pid"):
            np.testing.assert_array_equal(after[key], b[key], err_msg=key)
    kd.clean()


def test_random_grid():
    g = Grid()
    init = T.InitConfig.from_buffer_copy(bytes(g.init))
    init.grid_type = 1
    LIBC.srand(1)
    kd, got = device_state(g, init)
    kd.clean()
    LIBC.srand(1)
    ref = restated(g, random=True)
    for key in ("pos", "vel", "type", "pid"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)


class Fill(Grid):
    def __init__(self):
        z = np.load(os.path.join(HERE, "golden", "mill_fill.npz"))
        self.n_w, self.n_p, self.n_d = int(z["n_w"]), int(z["n_p"]), int(z["n_d"])
        self.wobj = (T.WOBJ * 8).from_buffer_copy(z["wobj"].tobytes())
        self.pobj = (T.POBJ * 8).from_buffer_copy(z["pobj"].tobytes())
        self.dobj = (T.DOBJ * 32).from_buffer_copy(z["dobj"].tobytes())
        self.sim_info = T.SimulationInfo.from_buffer_copy(z["sim_info"].tobytes())
        self.init = T.InitConfig.from_buffer_copy(z["init"].tobytes())
        self.per = (ctypes.c_int * 8)(*[int(v) for v in z["per_object"]])
        self.sim_info.Num_ParticlesPerObject = ctypes.cast(self.per, ctypes.POINTER(ctypes.c_int))
        self.n = self.sim_info.Num_Particles


def restated_fill(g):
    """Set_Position_Fill_Mill (DeviceInterface.cu:708-1054) for a ball mill
    with lifters, float32 throughout, glibc rand() for the shuffle."""
    f = np.float32
    si, c, w = g.sim_info, g.init, g.wobj[0]
    xs = f(2.0 * g.pobj[0].radius)
    sx, sy, sz = f(0.001), f(0.001), f(0.0)
    radius = f(si.DObject_CylinderBoundR)
    x0 = f(xs + f(f(w.cyl_geo.radius) - radius))
    y = f(w.cyl_geo.radius)
    z0 = f(f(f(w.cyl_geo.center_bot_cap.z) + f(xs / f(2.0))) + sz)
    NX = int(np.floor(f(f(f(radius * f(2)) - xs) / f(xs + sx))))
    NZ = int(np.floor(f(f(w.cyl_geo.height) / f(xs + sz))))
    NY = int(np.ceil(f(g.n / f(NX * NZ))))
    pos = np.zeros((g.n, 3), np.float32)
    typ = np.zeros(g.n, np.uint32)
    pid = np.arange(g.n, dtype=np.int32)
    per = [g.per[i] for i in range(g.n_p)]
    count, sel = [0] * g.n_p, -1
    z = z0
    for yd in range(NY):
        for zd in range(NZ):
            x = x0
            for xd in range(NX):
                k = yd * NZ * NX + zd * NX + xd
                if k >= g.n:
                    break
                pos[k] = (x, y, z)
                sel = sel + 1 if sel + 1 < g.n_p else 0
                pty = sel
                if count[pty] >= per[pty]:
                    pty = next(i for i in range(g.n_p) if count[i] <= per[i] - 1)
                count[pty] += 1
                typ[k] = pty
                x = f(f(x + xs) + sx)
            z = f(f(z + xs) + sz)
        z = z0
        y = f(f(y + xs) + sy)
    for _ in range(g.n):
        a = LIBC.rand() % (g.n - 1)
        b = LIBC.rand() % (g.n - 1)
        typ[a], typ[b] = typ[b], typ[a]
        pid[a], pid[b] = pid[b], pid[a]
    clear = int(abs(int(np.ceil(f(f(f(2.0) * xs) / f(f(si.InitalDelta_t) * f(c.launch_Vel.y)))))))
    return dict(pos=pos, type=typ, pid=pid), NX * NZ, clear


def test_mill_fill_waves():
    """The mill filled by waves (grid type 2): the lattice, then three waves
    (10,100 steps) on oracle A's trajectory with the same wave control."""
    g = Fill()
    LIBC.srand(1)
    kd, got = device_state(g, g.init)
    LIBC.srand(1)
    ref, pack, clear = restated_fill(g)
    for key in ("pos", "type", "pid"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)
    assert pack == 45 and clear == 5000
    if bindings.ref_available():
        zero = np.zeros((g.n, 3), np.float32)
        R = bindings.RefHost()
        R.init(g.sim_info, g.wobj, g.n_w, g.pobj, g.n_p, g.dobj, g.n_d, threads=4, capture=False)
        R.set_state(ref["pos"], zero, zero, ref["type"], ref["pid"])
        R.set_fill(pack, clear)
        steps = 2 * (clear + 1) + 99
        assert R.step(steps) == 0
        for _ in range(steps):
            kd.IDevice_DEM_UpdateSim()
        after = {k: np.zeros((g.n, 3), np.float32) for k in ("pos", "vel", "avel", "acc")}
        after["type"] = np.zeros(g.n, np.uint32)
        after["pid"] = np.zeros(g.n, np.int32)
        kd.IDevice_Get_System_State(after["pos"], None, after["vel"], after["avel"], after["acc"],
                                    after["type"], after["pid"])
        b = R.state()
        assert R.lib.refh_num_current() == 3 * pack
        for key in ("pos", "vel", "pid"):
            np.testing.assert_array_equal(after[key], b[key], err_msg=key)
    kd.clean()
