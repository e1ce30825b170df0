"""Canonical copies of boundary structs holding only the fields a run reads,
so that two parsers can be compared byte for byte although the reference's
parser leaves unused fields of its `new`-allocated arrays uninitialised
(V_02_2015/src/Input/KSimulationData.cpp:163, 238, 343).  TEST
INFRASTRUCTURE ONLY."""
import ctypes as C
import sys
import os

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "softx-d-15-00085_b200"))
from blaze import types as T  # noqa: E402


def _surface(dst, src):
    dst.num_vertex = src.num_vertex
    for k in range(max(0, min(src.num_vertex, 8))):
        dst.vertex_Order[k] = src.vertex_Order[k]
    dst.area = src.area
    dst.normal = src.normal
    dst.centroid = src.centroid
    dst.Tol = src.Tol


def wobj(src):
    d = T.WOBJ()
    d.surface_type = src.surface_type
    d.num_surfaces = src.num_surfaces
    d.num_vertex = src.num_vertex
    d.is_rotating = src.is_rotating
    for k in range(min(src.num_vertex, 16)):
        d.vertex[k] = src.vertex[k]
    if src.surface_type == 0:
        for j in range(min(src.num_surfaces, 16)):
            _surface(d.surfaces[j], src.surfaces[j])
    else:
        # field by field: the two bytes of padding after the bools, and
        # normal_cyl (never set by the reader), hold whatever the heap held
        for f in ("height", "radius", "has_top_cap", "has_bot_cap", "normal_top_cap",
                  "normal_bot_cap", "center_top_cap", "center_bot_cap", "AXIS"):
            setattr(d.cyl_geo, f, getattr(src.cyl_geo, f))
    if src.is_rotating:
        d.cyl_geo.AXIS = src.cyl_geo.AXIS
        d.cyl_geo.radius = src.cyl_geo.radius
    return bytes(d)


def pobj_sphere(src, n_types):
    d = T.POBJ()
    d.radius, d.mass = src.radius, src.mass
    for j in range(n_types):
        d.PP[j] = src.PP[j]
    for f in ("surface_Kn", "surface_Cn", "surface_Fric_static", "surface_Fric_kinetic",
              "Dsurface_Kn", "Dsurface_Cn", "Dsurface_Fric_static", "Dsurface_Fric_kinetic"):
        setattr(d, f, getattr(src, f))
    return bytes(d)


def pobj_poly(src, n_types):
    """A polyhedral particle object: geometry, mass, inertia tensor (as the
    parser leaves it, before the run setup scales it) and contact
    properties; face tolerances are never set for polyhedra."""
    d = T.POBJ()
    d.radius, d.mass, d.COM = src.radius, src.mass, src.COM
    d.num_vertex, d.num_faces, d.num_edges = src.num_vertex, src.num_faces, src.num_edges
    for k in range(min(src.num_vertex, 32)):
        d.vertex[k] = src.vertex[k]
        d.Local_Vertex[k] = src.Local_Vertex[k]
    for j in range(min(src.num_faces, 32)):
        _surface(d.face[j], src.face[j])
        d.face[j].Tol = 0.0
    for k in range(min(src.num_edges, 32)):
        d.edge[k] = src.edge[k]
    for g in range(9):
        d.InertiaT[g] = src.InertiaT[g]
    for j in range(n_types):
        d.PP[j] = src.PP[j]
    for f in ("surface_Kn", "surface_Cn", "surface_Fric_static", "surface_Fric_kinetic",
              "Dsurface_Kn", "Dsurface_Cn", "Dsurface_Fric_static", "Dsurface_Fric_kinetic"):
        setattr(d, f, getattr(src, f))
    return bytes(d)

def dobj(src):
    d = T.DOBJ()
    d.btype = src.btype
    if src.btype == 1:
        d.Axis = src.Axis
    d.boundR, d.COM = src.boundR, src.COM
    d.num_vertex, d.num_faces, d.num_edges = src.num_vertex, src.num_faces, src.num_edges
    for k in range(min(src.num_vertex, 8)):
        d.vertex[k] = src.vertex[k]
    for j in range(min(src.num_faces, 3)):
        _surface(d.faces[j], src.faces[j])
    for k in range(min(src.num_edges, 4)):
        d.edge[k] = src.edge[k]
    d.is_attached_DWorld, d.is_translating = src.is_attached_DWorld, src.is_translating
    if src.is_translating:
        d.velocity = src.velocity
    return bytes(d)
