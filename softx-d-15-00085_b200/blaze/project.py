"""Project-input mirror: reads a reference-format project tree into the POD
structs that the simulation-step boundary takes.

It restates, in order, the token reads and derived quantities of
  KSimulationData::KSimulationData       V_02_2015/src/Input/KSimulationData.cpp:27-700
  KSimulationData::ReadWObject           KSimulationData.cpp:704-883
  Set_SpringConstants*_KN / *_TC         KSimulationData.cpp:887-1071
  KSimulationData::ReadPObject_Sphere    KSimulationData.cpp:1076-1178
  KSimulationData::ReadPObject_Poly      KSimulationData.cpp:1183-1624
  KSimulationData::ReadDObject           KSimulationData.cpp:1650-1780
  KSimulationData::Repeat_Lifters        KSimulationData.cpp:1885-2028
  Set_SimInfo (headless part)            V_02_2015/src/main.cpp:469-832
  Read_FromFile (state files)            V_02_2015/src/Input/FileIO.h:327-652
Single-precision steps are evaluated in numpy float32 so every derived
float (normals, areas, centroids, masses, damping constants) equals the
reference parser's bit for bit; the CPU tests compare against the
reference's parser compiled on the host.

Errors the reference answers with exit(1) raise ProjectError here.
"""
import ctypes as C
import math
import os

import numpy as np

from . import types as T

F = np.float32
_libm = C.CDLL("libm.so.6")
_libm.cosf.restype = C.c_float
_libm.cosf.argtypes = [C.c_float]
_libm.sinf.restype = C.c_float
_libm.sinf.argtypes = [C.c_float]

PI = 2.0 * math.asin(1.0)


class ProjectError(RuntimeError):
    pass


# --------------------------------------------------------------------------
# float32 vector helpers (each operation rounded to float32, as compiled C)
def v3(x, y, z):
    return (F(x), F(y), F(z))


def vadd(a, b):
    return (F(a[0] + b[0]), F(a[1] + b[1]), F(a[2] + b[2]))


def vsub(a, b):
    return (F(a[0] - b[0]), F(a[1] - b[1]), F(a[2] - b[2]))


def vscale(s, a):
    s = F(s)
    return (F(s * a[0]), F(s * a[1]), F(s * a[2]))


def vdiv(a, s):
    s = F(s)
    return (F(a[0] / s), F(a[1] / s), F(a[2] / s))


def vdot(a, b):
    return F(F(F(a[0] * b[0]) + F(a[1] * b[1])) + F(a[2] * b[2]))


def vlen(a):
    return F(np.sqrt(vdot(a, a)))


def vcross(a, b):
    return (F(F(a[1] * b[2]) - F(a[2] * b[1])),
            F(F(a[2] * b[0]) - F(a[0] * b[2])),
            F(F(a[0] * b[1]) - F(a[1] * b[0])))


def tof3(f3):
    return (F(f3.x), F(f3.y), F(f3.z))


def setf3(dst, v):
    dst.x, dst.y, dst.z = float(v[0]), float(v[1]), float(v[2])


# --------------------------------------------------------------------------
class _Tokens:
    """Whitespace token stream with the semantics of `istream >> x`."""

    def __init__(self, path):
        if not os.path.isfile(path):
            raise ProjectError("file not found: %s" % path)
        with open(path, "r", errors="replace") as fh:
            self.tok = fh.read().split()
        self.i = 0
        self.path = path

    def s(self):
        if self.i >= len(self.tok):
            raise ProjectError("unexpected end of %s" % self.path)
        t = self.tok[self.i]
        self.i += 1
        return t

    def skip(self, n=1):
        for _ in range(n):
            self.s()

    def i_(self):
        t = self.s()
        try:
            return int(t)
        except ValueError:
            raise ProjectError("expected int, got %r in %s" % (t, self.path))

    def f(self):
        t = self.s()
        try:
            return float(t)
        except ValueError:
            raise ProjectError("expected number, got %r in %s" % (t, self.path))

    def f3(self):
        return v3(self.f(), self.f(), self.f())


def _cor_adjust(cor):
    # KSimulationData.cpp:908-911 and repeats: empirical COR correction.
    if 0.30 <= cor <= 0.90:
        cor -= 0.038080
    return cor


class Project:
    """A parsed project: the objects KSimulationData holds plus the
    SimulationInfo/InitConfig that Set_SimInfo derives from them."""

    def __init__(self):
        self.sim_info = T.SimulationInfo()
        self.init = T.InitConfig()
        self.wobj = (T.WOBJ * 8)()
        self.pobj = (T.POBJ * 8)()
        self.dobj = (T.DOBJ * 32)()
        self.n_w = self.n_p = self.n_d = 0
        self.num_lifters = 0
        self.per_object = (C.c_int * 16)()
        self.mill = T.Mill_Data()
        self.silo = T.Silo_Data()
        self.state_file = None
        self.sim_type = 0
        self.particle_type = 0
        self.force_spec = 1
        self.read_file = 0
        self.is_debug = 0
        self.world_size = v3(0, 0, 0)
        self.grid_origin = v3(0, 0, 0)
        self.grid_size = v3(0, 0, 0)
        self.delta_t = F(0)
        self.gravity = v3(0, 0, 0)
        self.is_rotation = 0
        self.roll_res = F(0)
        self.global_damp = F(0)
        self.vel_limit = F(0)
        self.num_particles = 0
        self.root = None
        self.stream_failed = False

    # ---------------------------------------------------------------- objects
    def _read_wobj(self, i, path):
        t = _Tokens(path)
        W = self.wobj[i]
        t.skip(2)  # Title
        t.skip(2)  # Descp
        t.skip(1)
        t.skip(1)
        W.num_vertex = t.i_()
        if W.num_vertex > 16:
            raise ProjectError("world object %d has %d vertices (max 16)" % (i, W.num_vertex))
        for j in range(W.num_vertex):
            t.skip(1)
            setf3(W.vertex[j], t.f3())
        t.skip(1)
        W.num_surfaces = t.i_()
        if W.num_surfaces > 16:
            raise ProjectError("world object %d has %d surfaces (max 16)" % (i, W.num_surfaces))
        for j in range(W.num_surfaces):
            acc = v3(0, 0, 0)
            idx = t.i_()
            t.skip(1)  # name
            W.surface_type = 1 if idx == -1 else 0
            S = W.surfaces[j]
            if W.surface_type == 0:
                t.skip(1)
                S.Tol = t.f()
                t.skip(1)
                S.num_vertex = t.i_()
                for f in range(S.num_vertex):
                    S.vertex_Order[f] = t.i_() - 1
                    acc = vadd(acc, tof3(W.vertex[S.vertex_Order[f]]))
            else:
                cg = W.cyl_geo
                t.skip(1)
                cg.radius = float(F(F(t.f()) * F(0.5)))
                t.skip(1)
                cg.height = t.f()
                t.skip(1)
                cg.has_top_cap = t.s() == "true"
                t.skip(1)
                cg.has_bot_cap = t.s() == "true"
                t.skip(1)
                setf3(cg.normal_top_cap, t.f3())
                t.skip(1)
                setf3(cg.normal_bot_cap, t.f3())
                t.skip(1)
                offset = t.f3()
                ones = v3(1, 1, 1)
                nb = tof3(cg.normal_bot_cap)
                setf3(cg.AXIS, vsub(ones, nb))
                cb = vadd(offset, vscale(cg.radius, vsub(ones, nb)))
                setf3(cg.center_bot_cap, cb)
                setf3(cg.center_top_cap, vadd(cb, (F(nb[0] * F(cg.height)), F(nb[1] * F(cg.height)),
                                                   F(nb[2] * F(cg.height)))))
            if W.surface_type == 0:
                vo = [tof3(W.vertex[S.vertex_Order[k]]) for k in range(S.num_vertex)]
                if S.num_vertex == 3:
                    V1 = vsub(vo[2], vo[0])
                    V2 = vsub(vo[1], vo[2])
                    n = vcross(V2, V1)
                    setf3(S.normal, vdiv(n, vlen(n)))
                    S.area = float(F(F(0.5) * vlen(n)))
                elif S.num_vertex == 4:
                    V1 = vsub(vo[1], vo[0])
                    V2 = vsub(vo[2], vo[1])
                    V3 = vsub(vo[3], vo[2])
                    V4 = vsub(vo[0], vo[3])
                    n = vcross(V2, V1)
                    setf3(S.normal, vdiv(n, vlen(n)))
                    S.area = float(F(F(F(0.5) * vlen(n)) + F(F(0.5) * vlen(vcross(V3, V4)))))
                setf3(S.centroid, vscale(F(F(1.0) / F(S.num_vertex)), acc))

    def _read_pobj_sphere(self, i, path, cor):
        t = _Tokens(path)
        P = self.pobj[i]
        t.skip(2)
        t.skip(2)
        t.skip(1)
        t.skip(1)
        P.radius = float(F(float(F(t.f())) * 0.5))
        t.skip(1)
        den = t.f()
        r = float(F(P.radius))
        P.mass = float(F((4.0 / 3.0) * 2.0 * math.asin(1.0) * math.pow(r, 3.0) * den * 1e-6))
        self._read_contact_props(t, i, cor)

    def _read_pobj_poly(self, i, path, cor):
        """KSimulationData::ReadPObject_Poly (KSimulationData.cpp:1219-1624)
        with Make_Particle_LocalInfo (1183-1215): vertices (Format 1 adds an
        offset, faces list comma-separated vertex numbers), centre of mass as
        the vertex mean, face centroids, normals from three face vertices,
        areas and volume by fans about the face centroid, mass from the
        density, the inertia tensor inverted element by element, body-frame
        vertices and the bounding radius, then the contact properties."""
        t = _Tokens(path)
        P = self.pobj[i]
        t.skip(2)
        t.skip(2)
        t.skip(1)
        fmt = t.i_()
        offset = v3(0, 0, 0)
        if fmt == 1:
            t.skip(1)
            offset = t.f3()
        t.skip(3)
        t.skip(1)
        nv = t.i_()
        if nv < 1 or nv > 32:
            raise ProjectError("polyhedron %d has %d vertices (1..32)" % (i, nv))
        P.num_vertex = nv
        verts = []
        size = [F(0), F(0), F(0)]
        acc = v3(0, 0, 0)
        for k in range(nv):
            if fmt == 0:
                t.skip(1)
                v = t.f3()
            else:
                v = vadd(t.f3(), offset)
            verts.append(v)
            setf3(P.vertex[k], v)
            for c in range(3):
                if v[c] > size[c]:
                    size[c] = v[c]
            acc = vadd(acc, v)
        setf3(self.init.p_size[i], size)
        com = vscale(F(F(1.0) / F(nv)), acc)
        setf3(P.COM, com)
        t.skip(1)
        nf = t.i_()
        if nf < 1 or nf > 32:
            raise ProjectError("polyhedron %d has %d faces (1..32)" % (i, nf))
        P.num_faces = nf
        vol = F(0)
        tot_area = None  # the reference's TotArea carries over between faces
        for j in range(nf):
            S = P.face[j]
            if fmt == 0:
                t.skip(2)
            fv = t.i_()
            if fv < 3 or fv > 8:
                raise ProjectError("polyhedron %d face %d has %d vertices (3..8)" % (i, j, fv))
            S.num_vertex = fv
            facc = v3(0, 0, 0)
            for f in range(fv):
                tok = t.s()
                if fmt == 1 and f < fv - 1:
                    tok = tok.rstrip(",")
                try:
                    o = int(tok) - 1
                except ValueError:
                    raise ProjectError("expected a vertex number, got %r in %s" % (tok, path))
                if o < 0 or o >= nv:
                    raise ProjectError("polyhedron %d face %d names vertex %d" % (i, j, o + 1))
                S.vertex_Order[f] = o
                facc = vadd(facc, verts[o])
            cen = vscale(F(F(1.0) / F(fv)), facc)
            setf3(S.centroid, cen)
            o = [S.vertex_Order[f] for f in range(fv)]

            def tet(a, b, c):
                return F(vdot(vsub(a, com), vcross(vsub(b, com), vsub(c, com))) / F(6.0))

            if fv == 3:
                n = vcross(vsub(verts[o[1]], verts[o[2]]), vsub(verts[o[2]], verts[o[0]]))
                setf3(S.normal, vdiv(n, vlen(n)))
                ad, bd, cd = (vsub(verts[o[k]], com) for k in range(3))
                vol = F(vol + F(F(np.sqrt(vdot(ad, vcross(bd, cd)))) / F(6.0)))
                if tot_area is None:
                    # the reference stores an uninitialised TotArea here
                    tot_area = F(F(0.5) * vlen(n))
            else:
                n = vcross(vsub(verts[o[2]], verts[o[3]]), vsub(verts[o[3]], verts[o[0]]))
                setf3(S.normal, vdiv(n, vlen(n)))
                tot_area = F(F(0.5) * vlen(vcross(vsub(verts[o[fv - 1]], cen),
                                                  vsub(verts[o[0]], cen))))
                vol = F(vol + tet(verts[o[fv - 1]], verts[o[0]], cen))
                for tr in range(fv - 1):
                    vol = F(vol + tet(verts[o[tr]], verts[o[tr + 1]], cen))
                    tot_area = F(tot_area + F(F(0.5) * vlen(vcross(vsub(verts[o[tr]], cen),
                                                                   vsub(verts[o[tr + 1]], cen)))))
            S.area = float(tot_area)
        t.skip(1)
        ne = t.i_()
        if ne < 0 or ne > 32:
            raise ProjectError("polyhedron %d has %d edges (0..32)" % (i, ne))
        P.num_edges = ne
        for k in range(ne):
            a, b = t.i_() - 1, t.i_() - 1
            if not (0 <= a < nv and 0 <= b < nv):
                raise ProjectError("polyhedron %d edge %d names a missing vertex" % (i, k))
            P.edge[k].point_vindex[0] = a
            P.edge[k].point_vindex[1] = b
        t.skip(3)
        t.skip(1)
        density = F(t.f())
        P.mass = float(F(float(F(density * vol)) * 1e-6))
        t.skip(1)
        for k in range(9):
            x = F(t.f())
            P.InertiaT[k] = float(F(1.0 / float(x))) if x > 0.0 else float(x)
        rad = F(0)
        for k in range(nv):
            lv = vsub(verts[k], com)
            setf3(P.Local_Vertex[k], lv)
            d = vlen(lv)
            if d > rad:
                rad = d
        P.radius = float(rad)
        t.skip(3)
        self._read_contact_props(t, i, cor)

    def _read_contact_props(self, t, i, cor):
        """The contact-property blocks shared by sphere and polyhedron
        objects (KSimulationData.cpp:1100-1175, 1543-1620): particle, surface
        and volume-object restitution with Kn (KN mode) or contact time (TC
        mode), friction coefficients, and the surface damping derived from
        them."""
        P = self.pobj[i]
        if self.force_spec == 0:
            t.skip(1)
            t.skip(1); cor[i] = t.f()
            t.skip(1); self._tc_pp = t.f()
            t.skip(1); P.PP[0].Fric_static = t.f()
            t.skip(1); P.PP[0].Fric_kinetic = t.f()
            t.skip(1)
            t.skip(1); cor_s = t.f()
            t.skip(1); tc_ps = t.f()
            t.skip(1); P.surface_Fric_static = t.f()
            t.skip(1); P.surface_Fric_kinetic = t.f()
            tc_ps *= float(self.delta_t)
            self._tc_pp *= float(self.delta_t)
            m = float(F(P.mass))
            c = _cor_adjust(cor_s)
            P.surface_Cn = 2.0 * m * (-math.log(c) / tc_ps)
            P.surface_Kn = (m / (tc_ps * tc_ps)) * (math.log(c) * math.log(c) + PI * PI)
            t.skip(1)
            t.skip(1); cor_d = t.f()
            t.skip(1); tc_pd = t.f()
            t.skip(1); P.Dsurface_Fric_static = t.f()
            t.skip(1); P.Dsurface_Fric_kinetic = t.f()
            tc_pd *= float(self.delta_t)
            c = _cor_adjust(cor_d)
            P.Dsurface_Cn = 2.0 * m * (-math.log(c) / tc_pd)
            P.Dsurface_Kn = (m / (tc_pd * tc_pd)) * (math.log(c) * math.log(c) + PI * PI)
        else:
            if i >= 6:
                raise ProjectError("KN mode supports at most 6 particle types (PP[6])")
            t.skip(1)
            t.skip(1); cor[i] = t.f()
            t.skip(1); P.PP[i].Kn = t.f()
            t.skip(1); P.PP[i].Fric_static = t.f()
            t.skip(1); P.PP[i].Fric_kinetic = t.f()
            t.skip(1)
            t.skip(1); cor_s = t.f()
            t.skip(1); P.surface_Kn = t.f()
            t.skip(1); P.surface_Fric_static = t.f()
            t.skip(1); P.surface_Fric_kinetic = t.f()
            m = float(F(P.mass))
            if cor_s < 1.0:
                c = _cor_adjust(cor_s)
                L = math.log(c)
                P.surface_Cn = -2.0 * L * math.sqrt(float(F(P.surface_Kn)) * m) / math.sqrt(L * L + PI * PI)
            else:
                P.surface_Cn = 0.0
            t.skip(1)
            t.skip(1); cor_d = t.f()
            t.skip(1); P.Dsurface_Kn = t.f()
            t.skip(1); P.Dsurface_Fric_static = t.f()
            t.skip(1); P.Dsurface_Fric_kinetic = t.f()
            if cor_d < 1.0:
                c = _cor_adjust(cor_d)
                L = math.log(c)
                P.Dsurface_Cn = -2.0 * L * math.sqrt(float(F(P.Dsurface_Kn)) * m) / math.sqrt(L * L + PI * PI)
            else:
                P.Dsurface_Cn = 0.0

    def _spring_pp_kn(self, i, j, cor_i, cor_j):
        # KSimulationData.cpp:955-1011
        Pi_, Pj = self.pobj[i], self.pobj[j]
        mi = float(F(Pi_.mass))
        if i == j:
            m = 1.0 / ((1.0 / mi) + (1.0 / mi))
            cor = cor_i
            if cor < 1.0:
                cor = _cor_adjust(cor)
                L = math.log(cor)
                Pi_.PP[j].Cn = -2.0 * L * math.sqrt(float(F(Pi_.PP[j].Kn)) * m) / math.sqrt(L * L + PI * PI)
            else:
                Pi_.PP[j].Cn = 0.0
        else:
            mj = float(F(Pj.mass))
            m = 1.0 / ((1.0 / mi) + (1.0 / mj))
            cor = _cor_adjust(0.5 * (cor_i + cor_j))
            Pi_.PP[j].Kn = float(F(F(0.5) * F(F(Pi_.PP[i].Kn) + F(Pj.PP[j].Kn))))
            Pi_.PP[j].Fric_static = 0.5 * (float(F(Pi_.PP[i].Fric_static)) + float(F(Pj.PP[j].Fric_static)))
            Pi_.PP[j].Fric_kinetic = 0.5 * (float(F(Pi_.PP[i].Fric_kinetic)) + float(F(Pj.PP[j].Fric_kinetic)))
            if cor < 1.0:
                L = math.log(cor)
                Pi_.PP[j].Cn = -2.0 * L * math.sqrt(float(F(Pi_.PP[j].Kn)) * m) / math.sqrt(L * L + PI * PI)
            else:
                Pi_.PP[j].Cn = 0.0

    def _spring_pp_tc(self, i, j, cor_i, cor_j):
        # KSimulationData.cpp:887-919
        Pi_, Pj = self.pobj[i], self.pobj[j]
        cor = 0.5 * (cor_i + cor_j)
        m = 1.0 / ((1.0 / float(F(Pi_.mass))) + (1.0 / float(F(Pj.mass))))
        cor = _cor_adjust(cor)
        if i == j:
            m = float(F(Pi_.mass))
        tc = self._tc_pp
        Pi_.PP[j].Cn = 2.0 * m * (-math.log(cor) / tc)
        Pi_.PP[j].Kn = (m / (tc * tc)) * (math.log(cor) * math.log(cor) + PI * PI)
        Pi_.PP[j].Fric_static = 0.5 * (float(F(Pi_.PP[0].Fric_static)) + float(F(Pj.PP[0].Fric_static)))
        Pi_.PP[j].Fric_kinetic = 0.5 * (float(F(Pi_.PP[0].Fric_kinetic)) + float(F(Pj.PP[0].Fric_kinetic)))

    def _read_dobj(self, i, path):
        t = _Tokens(path)
        D = self.dobj[i]
        t.skip(2)
        t.skip(2)
        t.skip(1)
        D.btype = t.i_()
        if D.btype == 1:
            t.skip(1)
            setf3(D.Axis, t.f3())
        t.skip(1)
        setf3(D.COM, t.f3())
        t.skip(1)
        D.boundR = t.f()
        t.skip(1)
        D.num_vertex = t.i_()
        if D.num_vertex > 0:
            for k in range(D.num_vertex):
                t.skip(1)
                setf3(D.vertex[k], t.f3())
            t.skip(1)
            D.num_faces = t.i_()
            for j in range(D.num_faces):
                acc = v3(0, 0, 0)
                t.skip(3)
                S = D.faces[j]
                S.Tol = t.f()
                t.skip(1)
                S.num_vertex = t.i_()
                for f in range(S.num_vertex):
                    S.vertex_Order[f] = t.i_() - 1
                    acc = vadd(acc, tof3(D.vertex[S.vertex_Order[f]]))
                setf3(S.centroid, vscale(F(F(1.0) / F(S.num_vertex)), acc))
                vo = [tof3(D.vertex[S.vertex_Order[k]]) for k in range(S.num_vertex)]
                if S.num_vertex == 3:
                    V1 = vsub(vo[2], vo[0])
                    V2 = vsub(vo[1], vo[2])
                    n = vcross(V1, V2)
                    setf3(S.normal, vdiv(n, vlen(n)))
                    S.area = float(F(F(0.5) * vlen(n)))
                elif S.num_vertex == 4:
                    V1 = vsub(vo[1], vo[0])
                    V2 = vsub(vo[2], vo[1])
                    V3 = vsub(vo[3], vo[2])
                    V4 = vsub(vo[0], vo[3])
                    n = vcross(V2, V1)
                    setf3(S.normal, vdiv(n, vlen(n)))
                    S.area = float(F(F(F(0.5) * vlen(n)) + F(F(0.5) * vlen(vcross(V3, V4)))))
            t.skip(1)
            D.num_edges = t.i_()
            for k in range(D.num_edges):
                D.edge[k].point_vindex[0] = (t.i_() - 1) & 0xFFFFFFFF
                D.edge[k].point_vindex[1] = (t.i_() - 1) & 0xFFFFFFFF

    def _make_new_lifter(self, about, index, d_index, angle):
        # KSimulationData.cpp:1885-1935 (cos/sin of a float angle: cosf/sinf)
        C.memmove(C.addressof(self.dobj[d_index]), C.addressof(self.dobj[index]), C.sizeof(T.DOBJ))
        D = self.dobj[d_index]
        ca = F(_libm.cosf(float(F(angle))))
        sa = F(_libm.sinf(float(F(angle))))
        for k in range(D.num_vertex):
            p = vsub(tof3(D.vertex[k]), about)
            x = F(F(ca * p[0]) + F(sa * p[1]))
            y = F(F(F(-sa) * p[0]) + F(ca * p[1]))
            setf3(D.vertex[k], vadd((x, y, p[2]), about))
        for j in range(D.num_faces):
            S = D.faces[j]
            acc = v3(0, 0, 0)
            for f in range(S.num_vertex):
                acc = vadd(acc, tof3(D.vertex[S.vertex_Order[f]]))
            setf3(S.centroid, vscale(F(F(1.0) / F(S.num_vertex)), acc))
            vo = [tof3(D.vertex[S.vertex_Order[k]]) for k in range(4)]
            V1 = vsub(vo[1], vo[0])
            V2 = vsub(vo[2], vo[1])
            V3 = vsub(vo[3], vo[2])
            V4 = vsub(vo[0], vo[3])
            n = vcross(V2, V1)
            setf3(S.normal, vdiv(n, vlen(n)))
            S.area = float(F(F(F(0.5) * vlen(n)) + F(F(0.5) * vlen(vcross(V3, V4)))))
        p = vsub(tof3(D.COM), about)
        x = F(F(ca * p[0]) + F(sa * p[1]))
        y = F(F(F(-sa) * p[0]) + F(ca * p[1]))
        setf3(D.COM, vadd((x, y, p[2]), about))

    def _repeat_lifters(self):
        # KSimulationData.cpp:1940-2028
        types = self.n_d
        num = self.num_lifters
        if num <= 0:
            return
        r = F(self.wobj[0].cyl_geo.radius)
        about = (r, r, F(0))
        theta = F(4.0 * math.asin(1.0) / float(F(num)))
        off = 0
        if types == 2:
            self._make_new_lifter(about, 1, 2, F(F(0.5) * theta))
            C.memmove(C.addressof(self.dobj[1]), C.addressof(self.dobj[2]), C.sizeof(T.DOBJ))
            off = 1
        dindex = 1 + off
        ee = 0
        for i in range(types):
            if i == 0:
                ee = 1
            for j in range(1, num - 1 + ee):
                self._make_new_lifter(about, i, dindex, F(theta * F(j)))
                dindex += 2 if types == 2 else 1
            dindex = 3
        self.n_d = types * num

    # ------------------------------------------------------------------ world
    @classmethod
    def load(cls, root, project, world, sim_2d=False):
        """Parse <root>/<project>/World/<world>.World and its objects."""
        self = cls()
        base = os.path.join(root, project)
        self.root = base
        t = _Tokens(os.path.join(base, "World", world + ".World"))
        t.skip(1); title = t.s()
        t.skip(1); self.force_spec = t.i_()
        t.skip(1); self.sim_type = t.i_()
        t.skip(1); self.particle_type = t.i_()
        t.skip(1); self.delta_t = F(t.f())
        self.is_debug = 1 if title == "UNIT_TEST" else 0
        if self.force_spec not in (0, 1):
            raise ProjectError("invalid force model (line 2)")
        if self.sim_type not in (0, 1, 2):
            raise ProjectError("invalid simulation mode (line 3)")
        if self.particle_type not in (0, 1):
            raise ProjectError("invalid particle type (line 4): mixed is not supported")
        t.skip(5)
        t.skip(1); self.n_w = t.i_()
        if self.n_w <= 0 or self.n_w > 8:
            raise ProjectError("invalid number of world objects (1..8)")
        for i in range(self.n_w):
            idx = t.i_()
            name = t.s()
            W = self.wobj[i]
            if idx == 99:
                W.is_rotating = True
                t.skip(1)
                ax = t.f3()
                setf3(W.cyl_geo.AXIS, ax)
                t.skip(1); self.mill.mill_RPM = t.f()
                t.skip(1); self.mill.total_revs = t.i_()
                W.cyl_geo.radius = float(max(max(ax[0], ax[1]), ax[2]))
                setf3(W.cyl_geo.AXIS, vdiv(ax, vlen(ax)))
            else:
                W.is_rotating = False
            self._read_wobj(i, os.path.join(base, "SurfaceObjects", name + ".WOBJ"))
        t.skip(3)
        t.skip(1); self.n_p = t.i_()
        if self.n_p <= 0 or self.n_p > 8:
            raise ProjectError("invalid number of particle objects (1..8)")
        cor = [0.0] * 6
        self._tc_pp = 0.0
        for i in range(self.n_p):
            t.skip(1)
            name = t.s()
            self.per_object[i] = t.i_()
            path = os.path.join(base, "ParticleObjects", name + ".POBJ")
            if self.particle_type == 1:
                self._read_pobj_poly(i, path, cor)
            else:
                self._read_pobj_sphere(i, path, cor)
        for i in range(self.n_p):
            for j in range(self.n_p):
                if self.force_spec == 0:
                    self._spring_pp_tc(i, j, cor[i], cor[j])
                else:
                    self._spring_pp_kn(i, j, cor[i], cor[j])
        t.skip(3)
        t.skip(1); self.n_d = t.i_()
        t.skip(1); self.num_lifters = t.i_()
        if self.n_d > 0:
            for i in range(self.n_d):
                idx = t.i_()
                name = t.s()
                D = self.dobj[i]
                if idx == 99:
                    D.is_attached_DWorld = False
                    D.is_translating = False
                elif idx == 98:
                    D.is_attached_DWorld = False
                    D.is_translating = True
                    t.skip(1)
                    setf3(D.velocity, t.f3())
                else:
                    D.is_attached_DWorld = True
                    D.is_translating = False
                sub = "LifterObjects" if self.sim_type == 1 else "VolumeObjects"
                self._read_dobj(i, os.path.join(base, sub, name + ".DOBJ"))
            if self.num_lifters > 0:
                self._repeat_lifters()
        t.skip(3)
        t.skip(1); self.num_particles = t.i_()
        t.skip(1); self.gravity = t.f3()
        t.skip(1)
        if sum(self.per_object[i] for i in range(self.n_p)) != self.num_particles:
            raise ProjectError("invalid number of particle objects")
        if float(self.delta_t) > 1e-1 or float(self.delta_t) < 0.0:
            raise ProjectError("invalid time step")
        t.skip(1); self.is_rotation = t.i_()
        t.skip(1); self.roll_res = F(t.f())
        t.skip(1); self.global_damp = F(t.f())
        t.skip(1); self.vel_limit = F(t.f())
        if float(self.roll_res) < 0.0:
            raise ProjectError("invalid rolling resistance")
        t.skip(3)
        t.skip(1); self.grid_origin = t.f3()
        t.skip(1); self.world_size = t.f3()
        t.skip(1); self.grid_size = t.f3()
        t.skip(3)
        t.skip(1); self.read_file = t.i_()
        if self.read_file == 1:
            t.skip(1); self.state_file = t.s()
            self.init.use_file = True
            self.init.grid_type = 0
        else:
            self.init.use_file = False
            t.skip(1); self.init.grid_type = t.i_()
            if self.init.grid_type < 2:
                t.skip(1); n = (t.i_(), t.i_(), t.i_())
                self.init.num.x, self.init.num.y, self.init.num.z = n
                t.skip(1); setf3(self.init.start, t.f3())
                t.skip(1); setf3(self.init.space, t.f3())
                t.skip(1); setf3(self.init.velocity[0], t.f3())
            else:
                t.skip(1); setf3(self.init.launch_Vel, t.f3())
                if self.sim_type != 1:
                    t.skip(1); setf3(self.init.fill_plane_start, t.f3())
                    t.skip(1); setf3(self.init.fill_plane_end, t.f3())
        # Output options and simulation-specific flags.  A token that does not
        # parse puts an istream into its fail state, after which every further
        # extraction leaves its target untouched; the reference's shipped silo
        # worlds rely on that (an integer read meets 'total_Time:').  Reading
        # stops at the first such token and the remaining fields keep their
        # defaults.
        try:
            t.skip(3)
            t.skip(1)
            if t.i_() > 0:
                color_type = t.i_()
                if color_type > 0:
                    t.f()
            t.skip(1); t.s()
            t.skip(1); t.s()
            t.skip(1); t.s()
            t.skip(1)
            if t.i_() > 0:
                t.s()
            t.skip(1); t.s()
            t.skip(1)
            if t.i_() == 1:
                t.s()
            t.skip(1); t.s()
            t.skip(1); t.s()
            t.skip(1)
            if self.sim_type == 1:
                t.skip(2)
                t.skip(1); self.mill.power_output_revs = t.i_()
                t.skip(1); self.mill.total_revs = t.i_()
                t.skip(1); self.mill.mill_RPM = t.f()
            elif self.sim_type == 2:
                t.skip(2)
                t.skip(1); self.silo.manual_hatch = t.i_() != 0
                t.skip(1); self.silo.measure_flow = t.i_() != 0
                self.silo.flow_steps = t.i_()
                t.skip(1); self.silo.kill_particle = t.i_() != 0
        except ProjectError:
            self.stream_failed = True
        self._set_sim_info(sim_2d)
        return self

    # ------------------------------------------------------------- setsiminfo
    def _set_sim_info(self, sim_2d):
        """Headless part of Set_SimInfo (main.cpp:469-832)."""
        si = self.sim_info
        si.Num_Particles = self.num_particles
        si.Num_WorldObjects = self.n_w
        si.Num_ParticleObjects = self.n_p
        si.Num_ParticlesPerObject = C.cast(self.per_object, C.POINTER(C.c_int))
        si.particle_type = self.particle_type
        si.InitalDelta_t = float(self.delta_t)
        setf3(si.Force_Field, self.gravity)
        si.Rotation = bool(self.is_rotation)
        si.Roll_Res = float(self.roll_res)
        si.Global_VisDamp = float(self.global_damp)
        si.Rotating_WObject = bool(self.wobj[0].is_rotating)
        si.Mode2D = bool(sim_2d)
        self.init.threads_perBlock = 1024
        if self.particle_type != 1:
            # sphere lattice step: the diameter (main.cpp:534-541); polyhedra
            # keep the largest vertex coordinates the parser found
            for i in range(self.n_p):
                d = float(F(F(self.pobj[i].radius) * F(2.0)))
                setf3(self.init.p_size[i], (d, d, d))
        setf3(si.cellSize, self.grid_size)
        setf3(si.worldOrigin, self.grid_origin)
        total = vsub(self.world_size, self.grid_origin)
        si.num_NNCells.x = int(math.ceil(float(F(total[0] / self.grid_size[0]))))
        si.num_NNCells.y = int(math.ceil(float(F(total[1] / self.grid_size[1]))))
        si.num_NNCells.z = int(math.ceil(float(F(total[2] / self.grid_size[2]))))
        si.unit_test = self.is_debug
        for i in range(self.n_p):
            P = self.pobj[i]
            r, m = F(P.radius), F(P.mass)
            scale = F(F(1.0) / F(F(F(F(0.4) * r) * r) * m))
            if self.particle_type == 0:
                P.InertiaT[0] = float(scale)
            else:
                # main.cpp:622-626: the inverted tensor scaled by 1/(0.4 m r^2)
                for g in range(9):
                    P.InertiaT[g] = float(F(scale * F(P.InertiaT[g])))
        si.Vel_Limit = float(self.vel_limit)
        if self.sim_type == 1:
            si.Simulation_Type = 1
            si.isMillSim = True
            si.EnergyCalc = self.mill.power_output_revs > 0
            rpm = F(self.mill.mill_RPM)
            self.mill.Num_Steps_PerRev = int(F(F(F(60.0) / rpm) / self.delta_t))
            self.mill.RadPerStep = float(-(F(F(F(rpm * F(2.0)) * F(PI)) / F(60.0))) * self.delta_t)
            vel_mill = abs((self.mill.RadPerStep / float(self.delta_t)) * float(F(self.wobj[0].cyl_geo.radius)) * 0.01)
            si.MillRotVel = -vel_mill
            if self.n_d > 0:
                si.DObject_CylinderBoundR = float(F(F(self.wobj[0].cyl_geo.radius) - F(F(2.0) * F(self.dobj[0].COM.y))))
                cb = self.wobj[0].cyl_geo.center_bot_cap
                setf3(si.cent, v3(cb.x, cb.y, 0.0))
        elif self.sim_type == 2:
            si.isMillSim = False
            hatch_h = F(self.wobj[self.n_w - 1].vertex[0].y)
            self.silo.hatch_height = float(hatch_h)
            si.Silo_Kill_Height = float(F(hatch_h - F(5.0)))
            si.Kill_Particles = bool(self.silo.kill_particle)
        elif si.Rotating_WObject:
            rpm = F(self.mill.mill_RPM)
            self.mill.RadPerStep = float(-(F(F(F(rpm * F(2.0)) * F(PI)) / F(60.0))) * self.delta_t)
            vel_mill = abs((self.mill.RadPerStep / float(self.delta_t)) *
                           (float(F(self.wobj[0].cyl_geo.radius)) - 100.0) * 0.01)
            si.MillRotVel = -vel_mill
        si.Integration_Type = 0
        si.use_symmetry = False
        si.sphere_orient = False
        if si.Rotating_WObject:
            si.Kill_Particles = False
        ncx, ncy, ncz = si.num_NNCells.x, si.num_NNCells.y, si.num_NNCells.z
        setf3(si.max_size, (F(F(ncx) * self.grid_size[0]), F(F(ncy) * self.grid_size[1]),
                            F(F(ncz) * self.grid_size[2])))
        si.use_hist = False

    # -------------------------------------------------------------- state i/o
    def read_state(self, fname=None):
        """Read a SpecType 1-4 state file (FileIO.h:327-652) into arrays in
        file order.  Returns a dict with pos, quat, vel, avel, acc, type, pid
        and the header values (time, spec_type)."""
        fname = fname or self.state_file
        return read_state_file(os.path.join(self.root, fname), self.num_particles,
                               self.particle_type, self.sim_type,
                               bool(self.wobj[0].is_rotating))


def _header_count(sim_type, rotating):
    # token pairs after "SpecType:" per simulation type (FileIO.h:348-496)
    if sim_type == 1:
        return 9
    if sim_type == 2:
        return 2
    if rotating:
        return 3
    return 1


def read_state_file(path, n, particle_type=0, sim_type=0, rotating=False):
    """Read a SpecType 1-4 state file (FileIO.h:327-652) into arrays in file
    order: pos, quat, vel, avel, acc, type, pid, spec_type, header."""
    with open(path, "r", errors="replace") as fh:
        text = fh.read()
    nl = text.find("\n")
    body = text[nl + 1:] if nl >= 0 else ""
    head = body.split(None, 2 + 2 * _header_count(sim_type, rotating))
    if len(head) < 2:
        raise ProjectError("truncated state file %s" % path)
    try:
        spec = int(head[1])
    except ValueError:
        raise ProjectError("bad SpecType in %s" % path)
    hdr_tok = head[2:2 + 2 * _header_count(sim_type, rotating)]
    hdr = {}
    names = {1: ["rev", "time", "revstate", "angle", "p0", "p1", "p2", "p3", "p4"],
             2: ["time", "num_rem"]}.get(sim_type, ["time", "steps", "angle"] if rotating else ["time"])
    for k, nm in enumerate(names):
        if 2 * k + 1 < len(hdr_tok):
            try:
                hdr[nm] = float(hdr_tok[2 * k + 1])
            except ValueError:
                raise ProjectError("bad header value in %s" % path)
    rest = head[-1] if len(head) == 3 + 2 * _header_count(sim_type, rotating) else ""
    poly = particle_type == 1
    cols = {1: 5 + (4 if poly else 0), 2: 11 + (4 if poly else 0),
            3: 11 + (4 if poly else 0), 4: 17 + (4 if poly else 0)}.get(spec)
    if cols is None:
        raise ProjectError("invalid SpecType %r" % spec)
    vals = np.array(rest.split()[:cols * n], dtype=np.float64)
    if vals.size < cols * n:
        raise ProjectError("state file %s holds fewer than %d particles" % (path, n))
    t = vals.reshape(n, cols)
    f32 = np.float32
    pos = t[:, 2:5].astype(f32)
    vel = np.zeros((n, 3), f32)
    acc = np.zeros((n, 3), f32)
    avel = np.zeros((n, 3), f32)
    quat = np.zeros((n, 4), f32)
    quat[:, 0] = 1.0
    c = 5
    if spec >= 2:
        vel = t[:, 5:8].astype(f32)
        c = 8
    if spec == 4:
        acc = t[:, 8:11].astype(f32)
        c = 11
    if poly:
        quat = t[:, c:c + 4].astype(f32)
        c += 4
    if spec >= 2:
        avel = t[:, c:c + 3].astype(f32)
    return dict(pos=pos, vel=vel, acc=acc, avel=avel, quat=quat, type=t[:, 1].astype(np.uint32),
                pid=t[:, 0].astype(np.int32), spec_type=spec, header=hdr)


def write_state_file(path, state, time=0.0, spec_type=3, sim_type=0,
                     header_line="#  P_ID   PType_ID   Pos   Vel   AngVel"):
    """Write a SpecType 3 state file (spheres) with the header line
    Read_FromFile expects for the simulation type (FileIO.h:348-496).
    Floats are written with 9 significant digits, which round-trips FP32."""
    pos, vel, avel = state["pos"], state["vel"], state["avel"]
    pid, ptype = state["pid"], state["type"]
    n = len(pid)
    with open(path, "w") as fh:
        fh.write(header_line + "\n")
        fh.write("Specfication_Detail: %d\n" % spec_type)
        if sim_type == 2:
            fh.write("  Time: %r NumRem: %d\n" % (float(time), n))
        elif sim_type == 1:
            fh.write(" RevNum: 0  Time: %r RevComplete: 0  RotAngle: 0.0  EParticle: 0 ELift 0 "
                     "EDrum: 0 ENorm: 0 EShear: 0\n" % float(time))
        else:
            fh.write("  Time: %r\n" % float(time))
        ints = np.stack([np.asarray(pid, np.int64), np.asarray(ptype, np.int64)], 1)
        fl = np.concatenate([np.asarray(pos, np.float32), np.asarray(vel, np.float32),
                             np.asarray(avel, np.float32)], 1).astype(np.float64)
        ia = np.char.mod("%d", ints)
        fa = np.char.mod("%.9g", fl)
        rows = np.concatenate([ia, fa], 1)
        fh.write("\n".join(" ".join(r) for r in rows.tolist()))
        fh.write("\n")
