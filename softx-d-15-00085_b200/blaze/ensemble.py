"""ctypes binding of the ensemble ABI (include/blaze_ens.h): many independent
sphere systems stepped together on one GPU with the linear or Hertz-Mindlin
contact law, tangential history spring, Coulomb cap and rolling friction.

Loading fails loudly when the library or a GPU is missing: there is no CPU
path in the product.
"""
import ctypes as C

import numpy as np

from .device import _check, _ptr, load as _load_lib

LAW_LINEAR = 1
LAW_HERTZ_MINDLIN = 2
LAW_REFERENCE = 3
WALL_PLANE = 0
WALL_TRIANGLE = 1
WALL_CYLINDER = 2


class Wall(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_float * 10)]


class System(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("origin", C.c_float * 3), ("cell", C.c_float), ("ncells", C.c_int * 3),
        ("gravity", C.c_float * 3), ("density", C.c_float), ("kn", C.c_float),
        ("kt_ratio", C.c_float), ("youngs", C.c_float), ("poisson", C.c_float),
        ("restitution", C.c_float), ("mu", C.c_float), ("mu_wall", C.c_float),
        ("mu_roll", C.c_float), ("wall0", C.c_int), ("nwalls", C.c_int), ("tri0", C.c_int),
        ("ntris", C.c_int), ("rot_point", C.c_float * 3), ("rot_axis", C.c_float * 3),
        ("rot_omega", C.c_float),
    ]


MAX_VERTS = 16
MAX_FACES = 28


class Shape(C.Structure):
    """blaze_shape: a convex hull in its body frame (centre of mass at the
    origin), triangular faces counter-clockwise seen from outside."""
    _fields_ = [("nverts", C.c_int), ("nfaces", C.c_int), ("density", C.c_float),
                ("verts", C.c_float * (3 * MAX_VERTS)), ("faces", C.c_int * (3 * MAX_FACES))]


class EnsOptions(C.Structure):
    _fields_ = [("law", C.c_int), ("dt", C.c_float), ("skin", C.c_float), ("max_nbr", C.c_int),
                ("use_graph", C.c_int), ("capture_forces", C.c_int), ("block", C.c_int)]


_bound = False


def load():
    global _bound
    lib = _load_lib()
    if not _bound:
        P = C.POINTER
        _f = P(C.c_float)
        _i = P(C.c_int)
        lib.blaze_ens_default_options.argtypes = [P(EnsOptions)]
        lib.blaze_ens_create.argtypes = [P(C.c_void_p), P(System), C.c_int, P(Wall), C.c_int,
                                         P(EnsOptions)]
        lib.blaze_ens_destroy.argtypes = [C.c_void_p]
        lib.blaze_ens_set_state.argtypes = [C.c_void_p, _f, _f, _f, _f]
        lib.blaze_ens_get_state.argtypes = [C.c_void_p, _f, _f, _f, _f, _i, _i]
        lib.blaze_ens_step.argtypes = [C.c_void_p, C.c_int]
        lib.blaze_ens_sync.argtypes = [C.c_void_p]
        lib.blaze_ens_set_params.argtypes = [C.c_void_p, P(System)]
        lib.blaze_ens_get_forces.argtypes = [C.c_void_p, _f, _f]
        lib.blaze_ens_num_rebuilds.argtypes = [C.c_void_p]
        lib.blaze_ens_device_state.argtypes = [C.c_void_p] + [P(C.c_void_p)] * 4
        lib.blaze_ens_last_launches.argtypes = [C.c_void_p]
        lib.blaze_ens_rebuild_kernels.argtypes = [C.c_void_p]
        lib.blaze_ens_adj_create.argtypes = [P(C.c_void_p), C.c_void_p, C.c_int, C.c_int]
        lib.blaze_ens_adj_forward.argtypes = [C.c_void_p]
        lib.blaze_ens_adj_backward.argtypes = [C.c_void_p, _f, _f, _f, _f, _f, _f,
                                               P(C.c_double)]
        lib.blaze_ens_adj_backward_window.argtypes = [C.c_void_p, C.c_int, _f, _f, _f, _f, _f,
                                                      _f, P(C.c_double)]
        lib.blaze_ens_adj_destroy.argtypes = [C.c_void_p]
        lib.blaze_ens_adj_profile.argtypes = [C.c_void_p, _f, _f, _f]
        lib.blaze_ens_adj_create_ex.argtypes = [P(C.c_void_p), C.c_void_p, C.c_int, C.c_int,
                                                C.c_longlong]
        lib.blaze_ens_adj_tape_info.argtypes = [C.c_void_p, P(C.c_ulonglong), P(C.c_int),
                                                P(C.c_ulonglong)]
        lib.blaze_ens_adj_create_tape.argtypes = [P(C.c_void_p), C.c_void_p, C.c_int, C.c_int,
                                                  C.c_ulonglong]
        lib.blaze_shape_mass_properties.argtypes = [P(Shape), P(C.c_double), P(C.c_double),
                                                    P(C.c_double), _f]
        lib.blaze_ens_set_polyhedra.argtypes = [C.c_void_p, P(Shape), C.c_int, _i, _f]
        lib.blaze_ens_get_orientations.argtypes = [C.c_void_p, _f]
        lib.blaze_ens_set_profile.argtypes = [C.c_void_p, C.c_int]
        lib.blaze_ens_profile.argtypes = [C.c_void_p, _f, _i]
        _bound = True
    return lib


def default_options(**kw):
    o = EnsOptions()
    load().blaze_ens_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def plane(normal, d):
    """Plane n . x = d, n (normalised here) pointing into the domain."""
    w = Wall()
    w.kind = WALL_PLANE
    n = np.asarray(normal, np.float64)
    n = n / np.linalg.norm(n)
    w.p[0], w.p[1], w.p[2], w.p[3] = float(n[0]), float(n[1]), float(n[2]), float(d)
    return w


def triangle(a, b, c):
    w = Wall()
    w.kind = WALL_TRIANGLE
    for k, v in enumerate(list(a) + list(b) + list(c)):
        w.p[k] = float(v)
    return w


def cylinder(point, axis, radius):
    """Cylinder wall (particles inside) through `point` along `axis`."""
    w = Wall()
    w.kind = WALL_CYLINDER
    ax = np.asarray(axis, np.float64)
    ax = ax / np.linalg.norm(ax)
    for k, v in enumerate(list(point) + list(ax) + [radius]):
        w.p[k] = float(v)
    return w


def shape(verts, faces, density):
    """A Shape from (V, 3) vertices (cm, about the centre of mass) and (F, 3)
    outward triangles; density in kg/cm^3."""
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    f = np.asarray(faces, np.int32).reshape(-1, 3)
    if len(v) > MAX_VERTS or len(f) > MAX_FACES:
        raise ValueError("shape: at most %d vertices and %d faces" % (MAX_VERTS, MAX_FACES))
    s = Shape()
    s.nverts, s.nfaces, s.density = len(v), len(f), float(density)
    for k, x in enumerate(v.reshape(-1)):
        s.verts[k] = float(x)
    for k, x in enumerate(f.reshape(-1)):
        s.faces[k] = int(x)
    return s


def mass_properties(s):
    """(mass kg, centre of mass (3,), inertia about it (3, 3) kg cm^2,
    bounding radius cm) of a Shape, from the library (FP64, no device)."""
    lib = load()
    m = C.c_double()
    com = np.zeros(3, np.float64)
    J = np.zeros(9, np.float64)
    rb = C.c_float()
    _check(lib.blaze_shape_mass_properties(C.byref(s), C.byref(m),
                                           com.ctypes.data_as(C.POINTER(C.c_double)),
                                           J.ctypes.data_as(C.POINTER(C.c_double)), C.byref(rb)),
           "blaze_shape_mass_properties")
    return m.value, com, J.reshape(3, 3), rb.value


class Ensemble:
    """Systems + walls on the GPU.  State arrays are (N, 3) float32 for all
    systems concatenated in system order."""

    def __init__(self, systems, walls, **options):
        self.lib = load()
        self.nsys = len(systems)
        self.systems = (System * self.nsys)(*systems)
        self.walls = (Wall * max(1, len(walls)))(*walls) if walls else (Wall * 1)()
        self.nwalls = len(walls)
        self.opts = default_options(**options)
        self.n = sum(s.n for s in systems)
        h = C.c_void_p()
        rc = self.lib.blaze_ens_create(C.byref(h), self.systems, self.nsys, self.walls,
                                       self.nwalls, C.byref(self.opts))
        _check(rc, "blaze_ens_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.blaze_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, pos, radius, vel=None, avel=None):
        c = np.ascontiguousarray
        n = self.n
        pos = c(pos, np.float32).reshape(n, 3)
        radius = c(radius, np.float32).reshape(n)
        vel = None if vel is None else c(vel, np.float32).reshape(n, 3)
        avel = None if avel is None else c(avel, np.float32).reshape(n, 3)
        _check(self.lib.blaze_ens_set_state(self.h, _ptr(pos, C.c_float), _ptr(radius, C.c_float),
                                            _ptr(vel, C.c_float), _ptr(avel, C.c_float)),
               "blaze_ens_set_state")

    def set_polyhedra(self, shapes, shape_of, quat):
        """After set_state: particle i (caller order) with shape_of[i] >= 0 is a
        polyhedron of shapes[shape_of[i]] oriented by quat[i] = (w, x, y, z)."""
        n = self.n
        arr = (Shape * len(shapes))(*shapes)
        so = np.ascontiguousarray(shape_of, np.int32).reshape(n)
        q = np.ascontiguousarray(quat, np.float32).reshape(n, 4)
        _check(self.lib.blaze_ens_set_polyhedra(self.h, arr, len(shapes), _ptr(so, C.c_int),
                                                _ptr(q, C.c_float)), "blaze_ens_set_polyhedra")

    def orientations(self):
        """(N, 4) orientations (w, x, y, z) in the current memory order."""
        q = np.zeros((self.n, 4), np.float32)
        _check(self.lib.blaze_ens_get_orientations(self.h, _ptr(q, C.c_float)),
               "blaze_ens_get_orientations")
        return q

    def step(self, n=1):
        return _check(self.lib.blaze_ens_step(self.h, int(n)), "blaze_ens_step")

    def sync(self):
        return _check(self.lib.blaze_ens_sync(self.h), "blaze_ens_sync")

    def state(self):
        n = self.n
        out = dict(pos=np.zeros((n, 3), np.float32), radius=np.zeros(n, np.float32),
                   vel=np.zeros((n, 3), np.float32), avel=np.zeros((n, 3), np.float32),
                   sys=np.zeros(n, np.int32), pid=np.zeros(n, np.int32))
        st = _check(self.lib.blaze_ens_get_state(
            self.h, _ptr(out["pos"], C.c_float), _ptr(out["radius"], C.c_float),
            _ptr(out["vel"], C.c_float), _ptr(out["avel"], C.c_float),
            _ptr(out["sys"], C.c_int), _ptr(out["pid"], C.c_int)), "blaze_ens_get_state")
        out["status"] = st
        return out

    def forces(self):
        n = self.n
        f = np.zeros((n, 3), np.float32)
        t = np.zeros((n, 3), np.float32)
        _check(self.lib.blaze_ens_get_forces(self.h, _ptr(f, C.c_float), _ptr(t, C.c_float)),
               "blaze_ens_get_forces")
        return f, t

    def set_params(self, systems):
        self.systems = (System * self.nsys)(*systems)
        _check(self.lib.blaze_ens_set_params(self.h, self.systems), "blaze_ens_set_params")

    def num_rebuilds(self):
        return _check(self.lib.blaze_ens_num_rebuilds(self.h), "blaze_ens_num_rebuilds")

    def device_state(self):
        ptrs = [C.c_void_p() for _ in range(4)]
        _check(self.lib.blaze_ens_device_state(self.h, *[C.byref(p) for p in ptrs]),
               "blaze_ens_device_state")
        return tuple(p.value for p in ptrs)

    def last_launches(self):
        return self.lib.blaze_ens_last_launches(self.h)

    def rebuild_kernels(self):
        return self.lib.blaze_ens_rebuild_kernels(self.h)

    def set_profile(self, on):
        _check(self.lib.blaze_ens_set_profile(self.h, int(bool(on))), "blaze_ens_set_profile")

    def profile(self):
        """(ms of re-sorts, polyhedron geometry, polyhedron step, sphere step)
        summed over the plain steps profiled, and their count."""
        ms = np.zeros(4, np.float32)
        n = C.c_int()
        _check(self.lib.blaze_ens_profile(self.h, _ptr(ms, C.c_float), C.byref(n)),
               "blaze_ens_profile")
        return ms.astype(np.float64), n.value


class Adjoint:
    """Reverse mode of an Ensemble over `nsteps` steps (linear law, plane
    walls): forward() steps the ensemble from its current state keeping a
    checkpoint every `segment` steps; backward() takes the cotangents of the
    final state (final memory order) and returns those of the initial state
    (its memory order) and of the law constants (nsys x 5: kn, kt, 2 beta,
    mu, mu_wall).

    tape_bytes: 0 keeps one segment on the tape (the forward records the
    last one; the backward recomputes the others from their checkpoints);
    a positive value is a budget in bytes; -1 takes 96 % of the free device
    memory less 4 GiB.  The trailing segments that fit are recorded by the
    forward and not recomputed."""

    def __init__(self, ens, nsteps, segment=100, tape_bytes=0, arena_bytes=None):
        """arena_bytes: the tape's arena size exactly, instead of tape_bytes."""
        self.ens = ens
        self.lib = ens.lib
        self.nsteps = int(nsteps)
        h = C.c_void_p()
        if arena_bytes is not None:
            _check(self.lib.blaze_ens_adj_create_tape(C.byref(h), ens.h, int(nsteps),
                                                      int(segment), int(arena_bytes)),
                   "blaze_ens_adj_create_tape")
        else:
            _check(self.lib.blaze_ens_adj_create_ex(C.byref(h), ens.h, int(nsteps),
                                                    int(segment), int(tape_bytes)),
                   "blaze_ens_adj_create_ex")
        self.h = h

    def tape_info(self):
        """(arena bytes, segments the last forward left on the tape, most pool
        bytes one recorded segment took)."""
        ab, pm = C.c_ulonglong(), C.c_ulonglong()
        m = C.c_int()
        _check(self.lib.blaze_ens_adj_tape_info(self.h, C.byref(ab), C.byref(m), C.byref(pm)),
               "blaze_ens_adj_tape_info")
        return ab.value, m.value, pm.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.blaze_ens_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self):
        return _check(self.lib.blaze_ens_adj_forward(self.h), "blaze_ens_adj_forward")

    def backward(self, gpos=None, gvel=None, gavel=None, window=None):
        """Cotangents of the final state -> (gx, gv, gw) of the initial
        state and the law constants (nsys x 5).  With `window`, only the
        last `window` steps are reversed (blaze_ens_adj_backward_window):
        the state cotangents are then those of the state `window` steps
        before the end."""
        n = self.ens.n
        c = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(n, 3)
        gpos, gvel, gavel = c(gpos), c(gvel), c(gavel)
        out = [np.zeros((n, 3), np.float32) for _ in range(3)]
        gc = np.zeros((self.ens.nsys, 5), np.float64)
        ptrs = [_ptr(gpos, C.c_float), _ptr(gvel, C.c_float), _ptr(gavel, C.c_float)] + \
            [_ptr(a, C.c_float) for a in out] + [gc.ctypes.data_as(C.POINTER(C.c_double))]
        if window is None:
            _check(self.lib.blaze_ens_adj_backward(self.h, *ptrs), "blaze_ens_adj_backward")
        else:
            _check(self.lib.blaze_ens_adj_backward_window(self.h, int(window), *ptrs),
                   "blaze_ens_adj_backward_window")
        return out[0], out[1], out[2], gc

    def profile(self):
        """Device ms of the last backward by phase: (restoring checkpoints,
        recomputing segments into the tape, reversing them)."""
        v = [C.c_float() for _ in range(3)]
        _check(self.lib.blaze_ens_adj_profile(self.h, *[C.byref(x) for x in v]),
               "blaze_ens_adj_profile")
        return tuple(x.value for x in v)


def beta2_of_e(e):
    """2 beta with beta = -ln e / sqrt(ln^2 e + pi^2) (damping from restitution)."""
    le = np.log(e)
    return 2.0 * (-le / np.sqrt(le * le + np.pi ** 2))


def dbeta2_de(e):
    le = np.log(e)
    return 2.0 * (-np.pi ** 2 / (e * (le * le + np.pi ** 2) ** 1.5))


def user_param_grads(gconst, systems):
    """Cotangents of (kn, kt_ratio, restitution, mu, mu_wall) per system from
    those of the law constants (kn, kt = kt_ratio kn, 2 beta(e), mu, mu_wall)."""
    out = np.zeros((len(systems), 5))
    for s, S in enumerate(systems):
        g = gconst[s]
        out[s, 0] = g[0] + g[1] * S.kt_ratio
        out[s, 1] = g[1] * S.kn
        out[s, 2] = g[2] * dbeta2_de(S.restitution)
        out[s, 3] = g[3]
        out[s, 4] = g[4]
    return out
