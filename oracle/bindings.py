"""ctypes bindings of the oracles.  TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product.

  RefHost   -- oracle A, oracle/_ref/libblaze_refhost.so: the reference's own
               kernels and project parser compiled as host C++.
  Restated  -- oracle/libdem_oracle_f32.so / _f64.so: this project's C
               restatement of the sphere path (dem_oracle.c), in FP32 (pinned
               bit-exact to oracle A) and FP64 (error reference).
"""
import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "softx-d-15-00085_b200"))
from blaze import types as T  # noqa: E402

REF_SO = os.path.join(HERE, "_ref", "libblaze_refhost.so")
F32_SO = os.path.join(HERE, "libdem_oracle_f32.so")
F64_SO = os.path.join(HERE, "libdem_oracle_f64.so")

_f = C.POINTER(C.c_float)
_u = C.POINTER(C.c_uint)
_i = C.POINTER(C.c_int)


def _p(a, ct):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ct))


class RefProject(C.Structure):
    _fields_ = [
        ("particle_type", C.c_int), ("sim_type", C.c_int), ("read_file", C.c_int),
        ("num_particles", C.c_int), ("n_w", C.c_int), ("n_p", C.c_int), ("n_d", C.c_int),
        ("num_lifters", C.c_int), ("is_debug", C.c_int), ("is_rotation", C.c_int),
        ("per_object", C.c_int * 16),
        ("delta_t", C.c_float), ("roll_res", C.c_float), ("global_damp", C.c_float),
        ("vel_limit", C.c_float),
        ("gravity", T.float3), ("grid_origin", T.float3), ("grid_size", T.float3),
        ("world_size", T.float3),
        ("filename", C.c_char * 256),
        ("mill", T.Mill_Data), ("silo", T.Silo_Data), ("init", T.InitConfig),
    ]


def ref_available():
    return os.path.isfile(REF_SO)


class RefHost:
    """Oracle A.  One simulation per process (the reference keeps its state
    in module globals, as DeviceInterface.cu does)."""

    _lib = None

    def __init__(self):
        if RefHost._lib is None:
            if not os.path.isfile(REF_SO):
                raise FileNotFoundError(REF_SO + " (build it with: make -C oracle ref)")
            lib = C.CDLL(REF_SO)
            lib.refh_sizeof.argtypes = [C.c_char_p]
            lib.refh_init.argtypes = [C.POINTER(T.SimulationInfo), C.POINTER(T.WOBJ), C.c_int,
                                      C.POINTER(T.POBJ), C.c_int, C.POINTER(T.DOBJ), C.c_int]
            lib.refh_set_state.argtypes = [_f, _f, _f, _f, _u, _i]
            lib.refh_get_state.argtypes = [_f, _f, _f, _f, _u, _i]
            lib.refh_get_forces.argtypes = [_f] * 6
            lib.refh_get_nlist.argtypes = [_u, _u]
            lib.refh_get_cells.argtypes = [_u, _u]
            lib.refh_get_energy.argtypes = [_f]
            lib.refh_get_lifter_hist.argtypes = [_i]
            lib.refh_update_wobj.argtypes = [C.POINTER(T.WOBJ), C.c_int]
            lib.refh_update_dobj.argtypes = [C.POINTER(T.DOBJ), C.c_int]
            lib.refh_open_hatch.argtypes = [C.POINTER(T.WOBJ), C.c_int]
            lib.refh_set_dobj_rotation.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int]
            lib.refh_get_dobj.argtypes = [C.POINTER(T.DOBJ), C.c_int]
            lib.refh_set_wobj_rotation.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int]
            lib.refh_set_dobj_translation.argtypes = [C.c_int, C.c_int]
            lib.refh_set_fill.argtypes = [C.c_int, C.c_int]
            lib.refh_get_wobj.argtypes = [C.POINTER(T.WOBJ), C.c_int]
            lib.refh_set_energy.argtypes = [_f]
            lib.refh_get_energy64.argtypes = [C.POINTER(C.c_double)]
            lib.refh_parse.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(RefProject),
                                       C.POINTER(T.WOBJ), C.c_int, C.POINTER(T.POBJ), C.c_int,
                                       C.POINTER(T.DOBJ), C.c_int]
            RefHost._lib = lib
        self.lib = RefHost._lib
        self.n = 0

    def sizeof(self, name):
        return self.lib.refh_sizeof(name.encode())

    def init(self, sim_info, wobj, n_w, pobj, n_p, dobj, n_d, threads=1, capture=True):
        rc = self.lib.refh_init(C.byref(sim_info), wobj, n_w, pobj, n_p, dobj, n_d)
        if rc:
            raise RuntimeError("refh_init failed: %d" % rc)
        self.n = sim_info.Num_Particles
        self.lib.refh_set_threads(int(threads))
        self.lib.refh_set_capture(1 if capture else 0)
        return self

    def set_cylinder_rotation(self, on):
        self.lib.refh_set_cylinder_rotation(1 if on else 0)

    def set_state(self, pos, vel, avel, ptype, pid, quat=None):
        c = np.ascontiguousarray
        self._keep = [c(pos, np.float32), None if quat is None else c(quat, np.float32),
                      c(vel, np.float32), c(avel, np.float32), c(ptype, np.uint32),
                      c(pid, np.int32)]
        k = self._keep
        self.lib.refh_set_state(_p(k[0], C.c_float), _p(k[1], C.c_float), _p(k[2], C.c_float),
                                _p(k[3], C.c_float), _p(k[4], C.c_uint), _p(k[5], C.c_int))

    def step(self, n=1):
        return self.lib.refh_step(int(n))

    def state(self):
        n = self.n
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        avel = np.zeros((n, 3), np.float32)
        quat = np.zeros((n, 4), np.float32)
        ptype = np.zeros(n, np.uint32)
        pid = np.zeros(n, np.int32)
        self.lib.refh_get_state(_p(pos, C.c_float), _p(quat, C.c_float), _p(vel, C.c_float),
                                _p(avel, C.c_float), _p(ptype, C.c_uint), _p(pid, C.c_int))
        return dict(pos=pos, vel=vel, avel=avel, quat=quat, type=ptype, pid=pid)

    def forces(self):
        n = self.n
        out = [np.zeros((n, 3), np.float32) for _ in range(6)]
        rc = self.lib.refh_get_forces(*[_p(a, C.c_float) for a in out])
        if rc:
            raise RuntimeError("forces not captured")
        keys = ["f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift"]
        return dict(zip(keys, out))

    def nlist(self):
        m = self.lib.refh_num_current()
        nn = np.zeros(m, np.uint32)
        lst = np.zeros((m, 32), np.uint32)
        self.lib.refh_get_nlist(_p(nn, C.c_uint), _p(lst, C.c_uint))
        return nn, lst

    def cells(self, ncell):
        s = np.zeros(ncell, np.uint32)
        e = np.zeros(ncell, np.uint32)
        self.lib.refh_get_cells(_p(s, C.c_uint), _p(e, C.c_uint))
        return s, e

    def energy(self):
        e = np.zeros(3, np.float32)
        self.lib.refh_get_energy(_p(e, C.c_float))
        return e

    def energy64(self):
        """The same tallies summed in FP64 (GetEnergy's units)."""
        e = np.zeros(3, np.float64)
        self.lib.refh_get_energy64(_p(e, C.c_double))
        return e

    def reset_energy(self):
        self.lib.refh_set_energy(None)

    def set_dobj_rotation(self, about_x, about_y, rad_per_step, on=True):
        """Turn the attached volume objects before every step, as the mill
        driver does (restated in ref_host/refhost_kernels.cpp)."""
        self.lib.refh_set_dobj_rotation(float(about_x), float(about_y), float(rad_per_step),
                                        1 if on else 0)

    def set_wobj_rotation(self, about_x, about_y, rad_per_step, on=True):
        self.lib.refh_set_wobj_rotation(float(about_x), float(about_y), float(rad_per_step),
                                        1 if on else 0)

    def set_fill(self, pack, clear):
        """Fill waves: `pack` particles join every clear + 1 steps."""
        self.lib.refh_set_fill(int(pack), int(clear))

    def set_dobj_translation(self, index, on=True):
        self.lib.refh_set_dobj_translation(int(index), 1 if on else 0)

    def wobj(self, n_w):
        w = (T.WOBJ * 8)()
        self.lib.refh_get_wobj(w, int(n_w))
        return w

    def dobj(self, n_d):
        d = (T.DOBJ * max(1, n_d))()
        self.lib.refh_get_dobj(d, int(n_d))
        return d

    @staticmethod
    def parse_isolated(projects_root, project, world):
        """The reference's parser in its own sanitizer-built process
        (oracle/_ref/refparse; polyhedral objects need it, see
        ref_host/refparse_main.cpp).  Same return values as parse()."""
        exe = os.path.join(HERE, "_ref", "refparse")
        tmp = tempfile.mkdtemp(prefix="blaze_refparse_")
        try:
            shutil.copytree(os.path.join(projects_root, project),
                            os.path.join(tmp, "Projects", project))
            os.makedirs(os.path.join(tmp, "run"))
            out = os.path.join(tmp, "out.bin")
            env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0")
            r = subprocess.run([exe, os.path.join(tmp, "run"), project, world, out],
                               env=env, capture_output=True, text=True, timeout=120)
            if r.returncode:
                raise RuntimeError("refparse failed (%d): %s" % (r.returncode, r.stderr[-400:]))
            raw = open(out, "rb").read()
            rp = RefProject.from_buffer_copy(raw[:C.sizeof(RefProject)])
            off = C.sizeof(RefProject)
            w = (T.WOBJ * 8).from_buffer_copy(raw[off:off + C.sizeof(T.WOBJ * 8)])
            off += C.sizeof(T.WOBJ * 8)
            p = (T.POBJ * 8).from_buffer_copy(raw[off:off + C.sizeof(T.POBJ * 8)])
            off += C.sizeof(T.POBJ * 8)
            d = (T.DOBJ * 32).from_buffer_copy(raw[off:off + C.sizeof(T.DOBJ * 32)])
            return rp, w, p, d
        finally:
            shutil.rmtree(tmp, ignore_errors=True)

    def parse(self, projects_root, project, world):
        """Parse with the reference's KSimulationData from a scratch copy of
        the project tree (the parser writes a log file into it)."""
        tmp = tempfile.mkdtemp(prefix="blaze_refparse_")
        try:
            shutil.copytree(os.path.join(projects_root, project),
                            os.path.join(tmp, "Projects", project))
            os.makedirs(os.path.join(tmp, "run"))
            rp = RefProject()
            w = (T.WOBJ * 8)()
            p = (T.POBJ * 8)()
            d = (T.DOBJ * 32)()
            rc = self.lib.refh_parse(os.path.join(tmp, "run").encode(), project.encode(),
                                     world.encode(), C.byref(rp), w, 8, p, 8, d, 32)
            if rc:
                raise RuntimeError("refh_parse failed: %d" % rc)
            return rp, w, p, d
        finally:
            shutil.rmtree(tmp, ignore_errors=True)


class DemLaw(C.Structure):
    _fields_ = [("model", C.c_int), ("kt_ratio", C.c_double), ("youngs", C.c_double),
                ("poisson", C.c_double), ("restitution", C.c_double), ("mu", C.c_double),
                ("mu_roll", C.c_double), ("skin", C.c_double), ("max_nbr", C.c_int)]


class Restated:
    """The C restatement (dem_oracle.c) in FP32 or FP64."""

    _libs = {}

    def __init__(self, precision="f32"):
        path = F32_SO if precision == "f32" else F64_SO
        if path not in Restated._libs:
            if not os.path.isfile(path):
                raise FileNotFoundError(path + " (build it with: make -C oracle)")
            lib = C.CDLL(path)
            _d = C.POINTER(C.c_double)
            lib.dem_create.restype = C.c_void_p
            lib.dem_create.argtypes = [C.POINTER(T.SimulationInfo), C.POINTER(T.WOBJ), C.c_int,
                                       C.POINTER(T.POBJ), C.c_int, C.POINTER(T.DOBJ), C.c_int]
            lib.dem_destroy.argtypes = [C.c_void_p]
            lib.dem_set_law.argtypes = [C.c_void_p, C.POINTER(DemLaw)]
            lib.dem_set_cylinder_rotation.argtypes = [C.c_void_p, C.c_int]
            lib.dem_set_state.argtypes = [C.c_void_p, _d, _d, _d, _u, _i]
            lib.dem_set_particle_props.argtypes = [C.c_void_p, _d, _d]
            lib.dem_step.argtypes = [C.c_void_p, C.c_int]
            lib.dem_num_current.argtypes = [C.c_void_p]
            lib.dem_status.argtypes = [C.c_void_p]
            lib.dem_get_state.argtypes = [C.c_void_p, _d, _d, _d, _u, _i]
            lib.dem_get_forces.argtypes = [C.c_void_p] + [_d] * 6
            lib.dem_get_nlist.argtypes = [C.c_void_p, _u, _u]
            lib.dem_get_energy.argtypes = [C.c_void_p, _d]
            lib.dem_update_wobj.argtypes = [C.c_void_p, C.POINTER(T.WOBJ), C.c_int]
            lib.dem_update_dobj.argtypes = [C.c_void_p, C.POINTER(T.DOBJ), C.c_int]
            lib.dem_set_mesh.argtypes = [C.c_void_p, _d, C.c_int, C.c_double, C.c_double, C.c_double]
            Restated._libs[path] = lib
        self.lib = Restated._libs[path]
        self.h = None
        self.max_nbr = 32

    def init(self, sim_info, wobj, n_w, pobj, n_p, dobj, n_d):
        self.h = self.lib.dem_create(C.byref(sim_info), wobj, n_w, pobj, n_p, dobj, n_d)
        if not self.h:
            raise RuntimeError("dem_create failed")
        self.n = sim_info.Num_Particles
        return self

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.dem_destroy(self.h)
            self.h = None

    def set_law(self, **kw):
        law = DemLaw(model=0, kt_ratio=2.0 / 7.0, max_nbr=32)
        for k, v in kw.items():
            setattr(law, k, v)
        self.max_nbr = law.max_nbr
        self.lib.dem_set_law(self.h, C.byref(law))

    def set_cylinder_rotation(self, on):
        self.lib.dem_set_cylinder_rotation(self.h, 1 if on else 0)

    def set_state(self, pos, vel, avel, ptype, pid):
        d = lambda a: np.ascontiguousarray(a, np.float64)
        self._keep = [d(pos), d(vel), d(avel), np.ascontiguousarray(ptype, np.uint32),
                      np.ascontiguousarray(pid, np.int32)]
        k = self._keep
        self.lib.dem_set_state(self.h, _p(k[0], C.c_double), _p(k[1], C.c_double),
                               _p(k[2], C.c_double), _p(k[3], C.c_uint), _p(k[4], C.c_int))

    def set_particle_props(self, radius=None, mass=None):
        if radius is None:
            self.lib.dem_set_particle_props(self.h, None, None)
            return
        self._kp = [np.ascontiguousarray(radius, np.float64), np.ascontiguousarray(mass, np.float64)]
        self.lib.dem_set_particle_props(self.h, _p(self._kp[0], C.c_double), _p(self._kp[1], C.c_double))

    def step(self, n=1):
        return self.lib.dem_step(self.h, int(n))

    def state(self):
        n = self.n
        pos, vel, avel = (np.zeros((n, 3)) for _ in range(3))
        ptype = np.zeros(n, np.uint32)
        pid = np.zeros(n, np.int32)
        self.lib.dem_get_state(self.h, _p(pos, C.c_double), _p(vel, C.c_double), _p(avel, C.c_double),
                               _p(ptype, C.c_uint), _p(pid, C.c_int))
        return dict(pos=pos, vel=vel, avel=avel, type=ptype, pid=pid)

    def forces(self):
        n = self.n
        out = [np.zeros((n, 3)) for _ in range(6)]
        self.lib.dem_get_forces(self.h, *[_p(a, C.c_double) for a in out])
        return dict(zip(["f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift"], out))

    def nlist(self):
        m = self.lib.dem_num_current(self.h)
        nn = np.zeros(m, np.uint32)
        lst = np.zeros((m, self.max_nbr), np.uint32)
        self.lib.dem_get_nlist(self.h, _p(nn, C.c_uint), _p(lst, C.c_uint))
        return nn, lst

    def status(self):
        return self.lib.dem_status(self.h)

    def energy(self):
        e = np.zeros(3)
        self.lib.dem_get_energy(self.h, _p(e, C.c_double))
        return e


ENS_F32_SO = os.path.join(HERE, "libens_oracle_f32.so")
ENS_F64_SO = os.path.join(HERE, "libens_oracle_f64.so")


class EnsRestated:
    """The C restatement of the ensemble path (ens_oracle.c) in FP32 or FP64.
    Takes the same System / Wall structs as the product's binding."""

    _libs = {}

    def __init__(self, systems, walls, law, dt, skin, max_nbr=32, precision="f32"):
        from blaze import ensemble as E
        path = ENS_F32_SO if precision == "f32" else ENS_F64_SO
        if path not in EnsRestated._libs:
            if not os.path.isfile(path):
                raise FileNotFoundError(path + " (build it with: make -C oracle)")
            lib = C.CDLL(path)
            _d = C.POINTER(C.c_double)
            lib.ens_create.restype = C.c_void_p
            lib.ens_create.argtypes = [C.POINTER(E.System), C.c_int, C.POINTER(E.Wall), C.c_int,
                                       C.c_int, C.c_double, C.c_double, C.c_int]
            lib.ens_destroy.argtypes = [C.c_void_p]
            lib.ens_set_params.argtypes = [C.c_void_p, C.POINTER(E.System)]
            lib.ens_set_state.argtypes = [C.c_void_p, _d, _d, _d, _d]
            lib.ens_step.argtypes = [C.c_void_p, C.c_int]
            lib.ens_get_state.argtypes = [C.c_void_p, _d, _d, _d, _d, _i, _i]
            lib.ens_get_forces.argtypes = [C.c_void_p, _d, _d]
            lib.ens_num_rebuilds.argtypes = [C.c_void_p]
            lib.ens_status.argtypes = [C.c_void_p]
            lib.ens_get_constants.argtypes = [C.c_void_p, C.c_int, _d]
            lib.ens_set_constants.argtypes = [C.c_void_p, C.c_int, _d]
            lib.ens_adj_record.argtypes = [C.c_void_p, C.c_int]
            lib.ens_adj_reverse.argtypes = [C.c_void_p, _d, _d, _d, _d, _d, _d, _d]
            lib.ens_set_polyhedra.argtypes = [C.c_void_p, C.POINTER(E.Shape), C.c_int, _i, _d]
            lib.ens_use_tri_lists.argtypes = [C.c_void_p, C.c_int]
            lib.ens_get_orientations.argtypes = [C.c_void_p, _d]
            EnsRestated._libs[path] = lib
        self.lib = EnsRestated._libs[path]
        self.nsys = len(systems)
        self._sys = (E.System * self.nsys)(*systems)
        self._walls = (E.Wall * max(1, len(walls)))(*walls) if walls else (E.Wall * 1)()
        self.n = sum(s.n for s in systems)
        self.h = self.lib.ens_create(self._sys, self.nsys, self._walls, len(walls), int(law),
                                     float(dt), float(skin), int(max_nbr))

    def close(self):
        if self.h:
            self.lib.ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, systems):
        from blaze import ensemble as E
        self._sys = (E.System * self.nsys)(*systems)
        self.lib.ens_set_params(self.h, self._sys)

    def set_state(self, pos, radius, vel=None, avel=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        self._keep = [c(pos), c(radius), c(vel), c(avel)]
        self.lib.ens_set_state(self.h, *[_p(a, C.c_double) for a in self._keep])

    def set_polyhedra(self, shapes, shape_of, quat):
        """After set_state, as blaze_ens_set_polyhedra: particle i with
        shape_of[i] >= 0 is a polyhedron of shapes[shape_of[i]] (ensemble
        Shape structs) oriented by quat[i] = (w, x, y, z)."""
        from blaze import ensemble as E
        arr = (E.Shape * len(shapes))(*shapes)
        so = np.ascontiguousarray(shape_of, np.int32)
        q = np.ascontiguousarray(quat, np.float64)
        self._keep_poly = [arr, so, q]
        rc = self.lib.ens_set_polyhedra(self.h, arr, len(shapes), _p(so, C.c_int), _p(q, C.c_double))
        if rc != 0:
            raise ValueError("ens_set_polyhedra: %d" % rc)

    def use_tri_lists(self, on):
        """1 (default): the triangles of the particle's cell only; 0: every
        triangle of the system (the same contacts)."""
        self.lib.ens_use_tri_lists(self.h, int(bool(on)))

    def orientations(self):
        q = np.zeros((self.n, 4))
        self.lib.ens_get_orientations(self.h, _p(q, C.c_double))
        return q

    def step(self, n=1):
        return self.lib.ens_step(self.h, int(n))

    def state(self):
        n = self.n
        out = dict(pos=np.zeros((n, 3)), radius=np.zeros(n), vel=np.zeros((n, 3)),
                   avel=np.zeros((n, 3)), sys=np.zeros(n, np.int32), pid=np.zeros(n, np.int32))
        self.lib.ens_get_state(self.h, _p(out["pos"], C.c_double), _p(out["radius"], C.c_double),
                               _p(out["vel"], C.c_double), _p(out["avel"], C.c_double),
                               _p(out["sys"], C.c_int), _p(out["pid"], C.c_int))
        out["status"] = self.lib.ens_status(self.h)
        return out

    def forces(self):
        n = self.n
        f = np.zeros((n, 3))
        t = np.zeros((n, 3))
        self.lib.ens_get_forces(self.h, _p(f, C.c_double), _p(t, C.c_double))
        return f, t

    def num_rebuilds(self):
        return self.lib.ens_num_rebuilds(self.h)

    def constants(self, s):
        """kn, kt, 2 beta, mu, mu_wall of system s, in working precision."""
        c = np.zeros(5)
        self.lib.ens_get_constants(self.h, int(s), _p(c, C.c_double))
        return c

    def set_constants(self, s, c5):
        c = np.ascontiguousarray(c5, np.float64)
        self.lib.ens_set_constants(self.h, int(s), _p(c, C.c_double))

    def adj_record(self, nsteps):
        return self.lib.ens_adj_record(self.h, int(nsteps))

    def adj_reverse(self, gx, gv, gw):
        """Cotangents of the final state (final memory order) -> cotangents
        of the recorded initial state (its memory order) and of the law
        constants (nsys x 5)."""
        n = self.n
        c = lambda a: np.ascontiguousarray(a, np.float64)
        gx, gv, gw = c(gx), c(gv), c(gw)
        out = [np.zeros((n, 3)) for _ in range(3)]
        th = np.zeros((self.nsys, 5))
        rc = self.lib.ens_adj_reverse(self.h, _p(gx, C.c_double), _p(gv, C.c_double),
                                      _p(gw, C.c_double), *[_p(a, C.c_double) for a in out],
                                      _p(th, C.c_double))
        if rc < 0:
            raise RuntimeError("ens_adj_reverse failed: %d" % rc)
        return out[0], out[1], out[2], th
