"""ctypes binding of libblaze_b200.so (include/blaze_dem.h).

`KDevice` mirrors the reference's wrapper class
(V_02_2015/src/Interface/KDevice.h:17-99): same method names, same argument
meaning, driving the module-level simulation of the C ABI's Part 1.
`Simulation` wraps the handle API (Part 2) for several independent
simulations and the options the reference does not have.

Loading fails loudly when the library or a GPU is missing: there is no CPU
path in the product.
"""
import ctypes as C
import os

import numpy as np

from . import types as T

LIB_PATH = os.environ.get("BLAZE_LIB") or os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                       "libblaze_b200.so")

STATUS_BITS = {1: "list_overflow", 2: "out_of_grid", 4: "non_finite", 8: "type_range",
               16: "timeout", 32: "poly_undefined", 64: "stale_list", 128: "cell_too_small"}

_f = C.POINTER(C.c_float)
_u = C.POINTER(C.c_uint)
_i = C.POINTER(C.c_int)


class BlazeError(RuntimeError):
    pass


class Options(C.Structure):
    _fields_ = [("skin", C.c_float), ("max_nbr", C.c_int), ("wall_grid", C.c_int),
                ("use_graph", C.c_int), ("capture_forces", C.c_int), ("sync_each_step", C.c_int),
                ("fast_law", C.c_int)]


class StateHeader(C.Structure):
    """blaze_state_header (include/blaze_dem.h): the values the reference's
    state writer takes from its driver (FileIO.h:12-315)."""
    _fields_ = [("detail", C.c_int), ("sim_type", C.c_int), ("rotating_wobj", C.c_int),
                ("particle_type", C.c_int), ("fill_start", C.c_int), ("revflag", C.c_int),
                ("rev_number", C.c_int), ("num_rem", C.c_int), ("rot_steps", C.c_int),
                ("steps_per_rev", C.c_int), ("time", C.c_double), ("rot_angle", C.c_double),
                ("energy", C.c_float * 5), ("hatch_height", C.c_float), ("dt", C.c_float)]


def state_header(**kw):
    h = StateHeader()
    h.detail = 3
    for k, v in kw.items():
        if k == "energy":
            for q, e in enumerate(v):
                h.energy[q] = float(e)
        else:
            setattr(h, k, v)
    return h


def write_state_arrays(path, header, pos, vel=None, avel=None, acc=None, ptype=None, pid=None,
                       quat=None, pobj=None, n_p=0):
    """Write host arrays (memory order) in the reference's state-file format."""
    lib = load()
    c = np.ascontiguousarray
    n = len(pos)
    arrs = [c(pos, np.float32), None if quat is None else c(quat, np.float32),
            None if vel is None else c(vel, np.float32), None if avel is None else c(avel, np.float32),
            None if acc is None else c(acc, np.float32), c(ptype, np.uint32), c(pid, np.int32)]
    return _check(lib.blaze_write_state_arrays(
        path.encode(), C.byref(header), n, _ptr(arrs[0], C.c_float), _ptr(arrs[1], C.c_float),
        _ptr(arrs[2], C.c_float), _ptr(arrs[3], C.c_float), _ptr(arrs[4], C.c_float),
        _ptr(arrs[5], C.c_uint), _ptr(arrs[6], C.c_int), pobj, int(n_p)), "blaze_write_state_arrays")


_lib = None


def load():
    """Load the library once (raises BlazeError when it cannot)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise BlazeError("libblaze_b200.so not built (%s); run __graft_entry__.build()" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    lib.blaze_default_options.argtypes = [P(Options)]
    lib.blaze_create.argtypes = [P(C.c_void_p), P(T.WOBJ), C.c_int, P(T.POBJ), C.c_int, P(T.DOBJ),
                                 C.c_int, P(T.SimulationInfo), P(Options)]
    lib.blaze_destroy.argtypes = [C.c_void_p]
    lib.blaze_set_options.argtypes = [C.c_void_p, P(Options)]
    lib.blaze_set_cylinder_rotation.argtypes = [C.c_void_p, C.c_int]
    lib.blaze_set_dobj_rotation.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int]
    lib.blaze_write_state_arrays.argtypes = [C.c_char_p, P(StateHeader), C.c_int] + \
        [P(C.c_float)] * 5 + [P(C.c_uint), P(C.c_int), P(T.POBJ), C.c_int]
    lib.blaze_write_state.argtypes = [C.c_void_p, C.c_char_p, P(StateHeader)]
    lib.blaze_get_dobj.argtypes = [C.c_void_p, C.POINTER(T.DOBJ), C.c_int]
    lib.blaze_set_dobj_translation.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.blaze_set_wobj_rotation.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int]
    lib.blaze_get_wobj.argtypes = [C.c_void_p, C.POINTER(T.WOBJ), C.c_int]
    lib.blaze_get_energy.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.blaze_set_energy.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.blaze_set_state.argtypes = [C.c_void_p, _f, _f, _f, _u, _i]
    lib.blaze_get_state.argtypes = [C.c_void_p, _f, _f, _f, _u, _i]
    lib.blaze_set_state_ornt.argtypes = [C.c_void_p, _f, _f, _f, _f, _u, _i]
    lib.blaze_get_state_ornt.argtypes = [C.c_void_p, _f, _f, _f, _f, _u, _i]
    lib.blaze_step.argtypes = [C.c_void_p, C.c_int]
    lib.blaze_sync.argtypes = [C.c_void_p]
    lib.blaze_num_current.argtypes = [C.c_void_p]
    lib.blaze_num_rebuilds.argtypes = [C.c_void_p]
    lib.blaze_prepare_graphs.argtypes = [C.c_void_p]
    lib.blaze_device_view.argtypes = [C.c_void_p] + [P(C.c_void_p), P(C.c_void_p), P(C.c_int),
                                                     P(C.c_void_p)]
    lib.blaze_num_exact_blocks.argtypes = [C.c_void_p]
    lib.blaze_update_wobj.argtypes = [C.c_void_p, P(T.WOBJ), C.c_int]
    lib.blaze_update_dobj.argtypes = [C.c_void_p, P(T.DOBJ), C.c_int]
    lib.blaze_get_forces.argtypes = [C.c_void_p] + [_f] * 6
    lib.blaze_get_nlist.argtypes = [C.c_void_p, _u, _u]
    lib.blaze_device_state.argtypes = [C.c_void_p] + [P(C.c_void_p)] * 4
    lib.blaze_last_launches.argtypes = [C.c_void_p]
    lib.blaze_set_profile.argtypes = [C.c_void_p, C.c_int]
    lib.blaze_open_hatch.argtypes = [C.c_void_p]
    lib.blaze_rebuild_kernels.argtypes = [C.c_void_p]
    lib.blaze_profile.argtypes = [C.c_void_p, _f, _f, _i]
    lib.blaze_count_above.argtypes = [C.c_void_p, C.c_float, _i]
    lib.blaze_write_flow_line.argtypes = [C.c_char_p, C.c_double, C.c_int, C.c_int]
    lib.blaze_write_power_line.argtypes = [C.c_char_p, C.c_double, _f, C.c_int, C.c_float]
    lib.blaze_default_sim.restype = C.c_void_p
    lib.Device_Set_SimulationData.argtypes = [P(T.WOBJ), P(T.POBJ), P(T.DOBJ), P(T.SimulationInfo),
                                              C.c_int, C.c_int, C.c_int, P(T.InitConfig)]
    f3p = P(T.float3)
    qp = P(T.Quaterion)
    lib.Device_Set_Pos.argtypes = [f3p, qp, _u, _i]
    lib.Device_Set_Pos_Velocity.argtypes = [f3p, qp, f3p, f3p, _u, _i]
    lib.Device_Set_System_State.argtypes = [f3p, qp, f3p, f3p, f3p, _u, _i]
    lib.Device_Set_Tallys.argtypes = [_f]
    lib.Device_Get_System_State.argtypes = [f3p, qp, f3p, f3p, f3p, _u, _i]
    lib.Device_Get_P_Positions.argtypes = [f3p, qp, _u, _i]
    lib.Device_Get_P_Velocity.argtypes = [f3p, f3p, C.c_int, _u, _i]
    lib.Device_Get_W_Forces.argtypes = [f3p, f3p]
    lib.Device_Get_Energy.argtypes = [_f]
    lib.Device_Update_DObjectPostions.argtypes = [P(T.DOBJ)]
    lib.Device_Update_WorldObjectPostions.argtypes = [P(T.WOBJ)]
    lib.Device_OpenHatch.argtypes = [P(T.WOBJ), C.c_int]
    lib.Device_Reset_Energy.argtypes = [C.c_int]
    lib.drum_rotation.argtypes = [C.c_bool]
    _lib = lib
    return lib


def _check(rc, what):
    if rc < 0:
        raise BlazeError("%s failed: %d" % (what, rc))
    return rc


def _ptr(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


def decode_status(st):
    return [name for bit, name in STATUS_BITS.items() if st & bit]


def default_options(**kw):
    o = Options()
    load().blaze_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class _DeviceArray:
    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 2}


def device_array(ptr, n, width, typestr="<f4"):
    """A torch view (no copy) of n x width device values at `ptr` (e.g. a
    pointer from Simulation.device_state or device_view)."""
    import torch
    return torch.as_tensor(_DeviceArray(int(ptr), (int(n), int(width)), typestr), device="cuda")


class Simulation:
    """One simulation on the GPU (handle API)."""

    def __init__(self, project=None, *, sim_info=None, wobj=None, n_w=0, pobj=None, n_p=0,
                 dobj=None, n_d=0, **options):
        lib = load()
        if project is not None:
            sim_info, wobj, n_w = project.sim_info, project.wobj, project.n_w
            pobj, n_p, dobj, n_d = project.pobj, project.n_p, project.dobj, project.n_d
        self.lib = lib
        self.n = sim_info.Num_Particles
        self.n_d = int(n_d)
        self.n_w = int(n_w)
        self.poly = sim_info.particle_type == 1
        self.opts = default_options(**options)
        h = C.c_void_p()
        rc = lib.blaze_create(C.byref(h), wobj, n_w, pobj, n_p, dobj, n_d, C.byref(sim_info),
                              C.byref(self.opts))
        _check(rc, "blaze_create")
        self.h = h
        self.max_nbr = self.opts.max_nbr

    def close(self):
        if getattr(self, "h", None):
            self.lib.blaze_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, **kw):
        for k, v in kw.items():
            setattr(self.opts, k, v)
        self.max_nbr = self.opts.max_nbr
        _check(self.lib.blaze_set_options(self.h, C.byref(self.opts)), "blaze_set_options")

    def set_cylinder_rotation(self, on):
        _check(self.lib.blaze_set_cylinder_rotation(self.h, 1 if on else 0), "cylinder rotation")

    def set_dobj_rotation(self, about_x, about_y, rad_per_step, on=True):
        """Turn the volume objects attached to the drum by rad_per_step about
        (about_x, about_y) before every step, on the device (the mill
        driver's Rotate_VolObject_Inc)."""
        _check(self.lib.blaze_set_dobj_rotation(self.h, float(about_x), float(about_y),
                                                float(rad_per_step), 1 if on else 0),
               "blaze_set_dobj_rotation")

    def set_dobj_translation(self, index, on=True):
        """Move volume object `index` by its velocity times dt before every
        step, on the device (the driver's Translate_VolObject)."""
        _check(self.lib.blaze_set_dobj_translation(self.h, int(index), 1 if on else 0),
               "blaze_set_dobj_translation")

    def set_wobj_rotation(self, about_x, about_y, rad_per_step, on=True):
        """Turn the world objects marked is_rotating before every step, on the
        device (the driver's Rotate_WObject_inc)."""
        _check(self.lib.blaze_set_wobj_rotation(self.h, float(about_x), float(about_y),
                                                float(rad_per_step), 1 if on else 0),
               "blaze_set_wobj_rotation")

    def wobj(self):
        w = (T.WOBJ * 8)()
        _check(self.lib.blaze_get_wobj(self.h, w, self.n_w), "blaze_get_wobj")
        return w

    def dobj(self):
        d = (T.DOBJ * max(1, self.n_d))()
        _check(self.lib.blaze_get_dobj(self.h, d, self.n_d), "blaze_get_dobj")
        return d

    def write_state(self, path, **header):
        """The current state in the reference's state-file format
        (blaze_state_header fields as keywords)."""
        h = state_header(**header)
        return _check(self.lib.blaze_write_state(self.h, path.encode(), C.byref(h)),
                      "blaze_write_state")

    def energy(self):
        """Energy tallies (particle-particle, volume objects, world objects)
        in Device_Get_Energy's units, FP64."""
        e = np.zeros(3, np.float64)
        _check(self.lib.blaze_get_energy(self.h, _ptr(e, C.c_double)), "blaze_get_energy")
        return e

    def reset_energy(self):
        _check(self.lib.blaze_set_energy(self.h, None), "blaze_set_energy")

    def set_state(self, pos, vel=None, avel=None, ptype=None, pid=None, quat=None):
        """Positions (centres of mass), velocities, angular velocities,
        types, P_IDs and, for polyhedra, orientations (w, x, y, z)."""
        n = self.n
        c = np.ascontiguousarray
        pos = c(pos, np.float32).reshape(n, 3)
        vel = None if vel is None else c(vel, np.float32).reshape(n, 3)
        avel = None if avel is None else c(avel, np.float32).reshape(n, 3)
        quat = None if quat is None else c(quat, np.float32).reshape(n, 4)
        ptype = np.zeros(n, np.uint32) if ptype is None else c(ptype, np.uint32)
        pid = np.arange(n, dtype=np.int32) if pid is None else c(pid, np.int32)
        rc = self.lib.blaze_set_state_ornt(self.h, _ptr(pos, C.c_float), _ptr(quat, C.c_float),
                                           _ptr(vel, C.c_float), _ptr(avel, C.c_float),
                                           _ptr(ptype, C.c_uint), _ptr(pid, C.c_int))
        _check(rc, "blaze_set_state")

    def step(self, n=1):
        return _check(self.lib.blaze_step(self.h, int(n)), "blaze_step")

    def sync(self):
        return _check(self.lib.blaze_sync(self.h), "blaze_sync")

    def state(self):
        n = self.n
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        avel = np.zeros((n, 3), np.float32)
        ptype = np.zeros(n, np.uint32)
        pid = np.zeros(n, np.int32)
        quat = np.zeros((n, 4), np.float32) if self.poly else None
        st = _check(self.lib.blaze_get_state_ornt(self.h, _ptr(pos, C.c_float),
                                                  _ptr(quat, C.c_float), _ptr(vel, C.c_float),
                                                  _ptr(avel, C.c_float), _ptr(ptype, C.c_uint),
                                                  _ptr(pid, C.c_int)), "blaze_get_state")
        out = dict(pos=pos, vel=vel, avel=avel, type=ptype, pid=pid, status=st)
        if self.poly:
            out["quat"] = quat
        return out

    def forces(self):
        n = self.n
        out = [np.zeros((n, 3), np.float32) for _ in range(6)]
        _check(self.lib.blaze_get_forces(self.h, *[_ptr(a, C.c_float) for a in out]),
               "blaze_get_forces")
        return dict(zip(["f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift"], out))

    def nlist(self):
        n = self.n
        nn = np.zeros(n, np.uint32)
        lst = np.zeros((n, self.max_nbr), np.uint32)
        _check(self.lib.blaze_get_nlist(self.h, _ptr(nn, C.c_uint), _ptr(lst, C.c_uint)),
               "blaze_get_nlist")
        return nn, lst

    def num_current(self):
        return _check(self.lib.blaze_num_current(self.h), "blaze_num_current")

    def num_rebuilds(self):
        return _check(self.lib.blaze_num_rebuilds(self.h), "blaze_num_rebuilds")

    def prepare_graphs(self):
        """Instantiate the CUDA graphs graph stepping will launch (no capture
        then happens inside later steps)."""
        _check(self.lib.blaze_prepare_graphs(self.h), "blaze_prepare_graphs")

    def count_above(self, height):
        """Particles of the current run whose centre is above `height`
        (the silo's remaining count, main.cpp:253-276), counted on the device."""
        n = C.c_int()
        _check(self.lib.blaze_count_above(self.h, float(height), C.byref(n)), "blaze_count_above")
        return n.value

    def num_exact_blocks(self):
        return _check(self.lib.blaze_num_exact_blocks(self.h), "blaze_num_exact_blocks")

    def update_wobj(self, wobj, n_w):
        _check(self.lib.blaze_update_wobj(self.h, wobj, n_w), "blaze_update_wobj")

    def update_dobj(self, dobj, n_d):
        _check(self.lib.blaze_update_dobj(self.h, dobj, n_d), "blaze_update_dobj")

    def device_state(self):
        """(pos4, vel4, angv4, stream) device pointers as ints."""
        ptrs = [C.c_void_p() for _ in range(4)]
        _check(self.lib.blaze_device_state(self.h, *[C.byref(p) for p in ptrs]), "device_state")
        return tuple(p.value for p in ptrs)

    def device_view(self):
        """(pos4, ornt4 or None, n, stream): the headless view buffer, device
        pointers as ints (blaze_device_view)."""
        pos, orn, st = C.c_void_p(), C.c_void_p(), C.c_void_p()
        n = C.c_int()
        _check(self.lib.blaze_device_view(self.h, C.byref(pos), C.byref(orn), C.byref(n),
                                          C.byref(st)), "blaze_device_view")
        return pos.value, orn.value, n.value, st.value

    def last_launches(self):
        return self.lib.blaze_last_launches(self.h)

    def rebuild_kernels(self):
        return self.lib.blaze_rebuild_kernels(self.h)

    def open_hatch(self):
        _check(self.lib.blaze_open_hatch(self.h), "blaze_open_hatch")

    def set_profile(self, on):
        _check(self.lib.blaze_set_profile(self.h, 1 if on else 0), "blaze_set_profile")

    def profile(self):
        """(ms in re-sort + list phases, ms in the fused step kernel, steps)."""
        a, b, n = C.c_float(), C.c_float(), C.c_int()
        _check(self.lib.blaze_profile(self.h, C.byref(a), C.byref(b), C.byref(n)), "blaze_profile")
        return a.value, b.value, n.value


class KDevice:
    """Mirror of the reference's KDevice (KDevice.h:17-99) over the C ABI's
    module-level simulation.  Arrays are numpy float32 (N,3), uint32, int32."""

    def __init__(self, worldObject, particleObject, dynamicObject, num_worldObjects,
                 num_particleObjects, num_dynamicObjects, simInfo, h_PosConfig=None):
        self.lib = load()
        self.n = simInfo.Num_Particles
        init = h_PosConfig if h_PosConfig is not None else T.InitConfig()
        rc = self.lib.Device_Set_SimulationData(worldObject, particleObject, dynamicObject,
                                                C.byref(simInfo), num_worldObjects,
                                                num_particleObjects, num_dynamicObjects,
                                                C.byref(init))
        _check(rc, "Device_Set_SimulationData")

    @staticmethod
    def _f3(a):
        return None if a is None else a.ctypes.data_as(C.POINTER(T.float3))

    @staticmethod
    def _q(a):
        """Orientations, float32 (N, 4) as (w, x, y, z), or None."""
        return None if a is None else a.ctypes.data_as(C.POINTER(T.Quaterion))

    def clean(self):
        return self.lib.Device_Clean()

    def IDevice_DEM_UpdateSim(self):
        return _check(self.lib.Device_DEM_UpdateSim(), "Device_DEM_UpdateSim")

    def IDevice_Mill_reset_energy(self, value):
        return self.lib.Device_Reset_Energy(int(value))

    def IDevice_UpdateVolObjectPositions(self, h_DynamicOBJ):
        return _check(self.lib.Device_Update_DObjectPostions(h_DynamicOBJ), "update DOBJ")

    def IDevice_UpdateWorldObjects(self, h_WorldOBJ):
        return _check(self.lib.Device_Update_WorldObjectPostions(h_WorldOBJ), "update WOBJ")

    def IDevice_OpenHatch(self, h_WorldOBJ, h_Num_WorldOBJ):
        return _check(self.lib.Device_OpenHatch(h_WorldOBJ, h_Num_WorldOBJ), "open hatch")

    def IDevice_Set_Tallys(self, h_Tallys):
        a = np.ascontiguousarray(h_Tallys, np.float32)
        return self.lib.Device_Set_Tallys(_ptr(a, C.c_float))

    def IDevice_drum_rotation(self, on):
        return _check(self.lib.drum_rotation(bool(on)), "drum_rotation")

    def IDevice_Get_System_State(self, h_pos, h_Ornt, h_vel, h_Avel, h_acc, h_type, h_pid):
        return _check(self.lib.Device_Get_System_State(
            self._f3(h_pos), self._q(h_Ornt), self._f3(h_vel), self._f3(h_Avel), self._f3(h_acc),
            _ptr(h_type, C.c_uint), _ptr(h_pid, C.c_int)), "Device_Get_System_State")

    def IDevice_Get_Positions(self, h_pos, h_Quart_ornt, h_type, P_ID):
        return _check(self.lib.Device_Get_P_Positions(self._f3(h_pos), self._q(h_Quart_ornt),
                                                      _ptr(h_type, C.c_uint), _ptr(P_ID, C.c_int)),
                      "Device_Get_P_Positions")

    def IDevice_Get_Particle_Velocity(self, H_Vel, H_Rvel, flag, h_type, P_ID):
        return _check(self.lib.Device_Get_P_Velocity(self._f3(H_Vel), self._f3(H_Rvel), int(flag),
                                                     _ptr(h_type, C.c_uint), _ptr(P_ID, C.c_int)),
                      "Device_Get_P_Velocity")

    def IDevice_Get_W_Forces(self, WallForces, WallContact_Point=None):
        return self.lib.Device_Get_W_Forces(self._f3(WallForces), self._f3(WallContact_Point))

    def IDevice_Get_Energy(self, Energy):
        return self.lib.Device_Get_Energy(_ptr(Energy, C.c_float))

    def IDevice_Set_ParticleSystem_State(self, h_pos, h_Ornt, h_vel, h_Avel, h_acc, h_type, h_pid):
        return _check(self.lib.Device_Set_System_State(
            self._f3(h_pos), self._q(h_Ornt), self._f3(h_vel), self._f3(h_Avel), self._f3(h_acc),
            _ptr(h_type, C.c_uint), _ptr(h_pid, C.c_int)), "Device_Set_System_State")

    def IDevice_Set_ParticleSystem_Pos(self, h_pos, h_Ornt, h_type, h_pid):
        return _check(self.lib.Device_Set_Pos(self._f3(h_pos), self._q(h_Ornt),
                                              _ptr(h_type, C.c_uint), _ptr(h_pid, C.c_int)),
                      "Device_Set_Pos")

    def IDevice_Set_ParticleSystem_PosV(self, h_pos, h_Ornt, h_vel, h_Avel, h_type, h_pid):
        return _check(self.lib.Device_Set_Pos_Velocity(
            self._f3(h_pos), self._q(h_Ornt), self._f3(h_vel), self._f3(h_Avel),
            _ptr(h_type, C.c_uint), _ptr(h_pid, C.c_int)), "Device_Set_Pos_Velocity")

    def IStart_Bin(self):
        return self.lib.Start_Bin()

    def IDevice_AddForce(self):
        return self.lib.Device_AddForce()

    def IDevice_SubForce(self):
        return self.lib.Device_SubForce()

    def IDevice_ZeroForce(self):
        return self.lib.Device_ZeroForce()
