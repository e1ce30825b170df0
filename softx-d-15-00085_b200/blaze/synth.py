"""Seeded synthetic workloads, written as reference-format project trees
(.World / .POBJ / .WOBJ and a SpecType-3 state file) so that every run goes
through the project-input path a user of the reference would use.

Units are the reference's: cm, kg, s (Kn in kg/s^2 has the same number in
SI and in these units).  All randomness is numpy default_rng(seed).

  box_project    10,000 monodisperse spheres in a closed cube
                 (the Particles_Box plain configuration)
  silo_project   polydisperse spheres in a cylindrical silo over a conical
                 hopper approximated by planar faces (reference-law variant
                 of the silo discharge configuration: at most 6 radius bins,
                 linear law, hopper faces within the 8 x 16 face capacity)
  poly_box_project
                 convex polyhedra (dodecahedra, cubes, hexagonal prisms) in
                 a closed box, every particle in contact from the start
  silo_full_ensemble
                 the silo discharge in its full form (Hertz-Mindlin, rolling
                 friction, a 4,096-triangle hopper) as a one-system ensemble
  mill_project   polydisperse steel spheres in a ball-mill drum with end
                 plates and lifters turned with it (the ball-mill
                 configuration's sphere charge, reference path)
"""
import math
import os

import numpy as np

from .project import Project, write_state_file

_WORLD = """Title: "{title}"
ModelType(Specfic|0:TC_COR|1:KN_COR):     1
Simulation_Type(0=General,1=mill,2=silo): {sim_type}
Particle_Type(0=sphere,1=poly,2=mixed):   {ptype}
Delta_t(s):       {dt!r}
_________________________________________________
             1_Geometrical-Information
---------------------------------------
 1.1_World_Objects_(index__name)
---------------------------------------
Number: {n_w}
{wobj_lines}
---------------------------------------
 1.2_Particle_Objects_(index__name__number)
---------------------------------------
Number: {n_p}
{pobj_lines}
---------------------------------------
 1.3_Dynamic_Objects_(index__name)
---------------------------------------
{dobj_lines}
_________________________________________________
_________________________________________________
             2_Simulation_Setup
Num_Particles:    {n}
ForceField(cm/s^2): {g[0]!r} {g[1]!r} {g[2]!r}
---------------------------------------------
Rotation:         {rotation}
RollRes:          {roll_res!r}
GlobalDamp:       1.0
VelLimit:         0.0
_________________________________________________
_________________________________________________
            3_Spatial-Grid-Computation
Origin:       {origin[0]!r} {origin[1]!r} {origin[2]!r}
World_Size:   {world[0]!r} {world[1]!r} {world[2]!r}
Cell_Size:    {cell!r} {cell!r} {cell!r}
_________________________________________________
_________________________________________________
            4_Inital_Particle-Setup
Read_FromFile: 1
FileName: {state}
_________________________________________________
_________________________________________________
             5_Output_Options
Display:           0
View:              0
FPS:               50
GL_DEBUG           0
File_write(Steps): 0
Total_Time:        0.0
IS_Time_Limit:     0
IS_Energy_diss(steps): 0
IS_Wall_forces(steps): 0
_________________________________________________
{specific}"""

_POBJ = """Title: "{title}"
Descp: "synthetic"
Geometry_Specfications
Diameter: {diam!r}
Density:  {rho!r}
Particle_Particle
COR:       {cor!r}
Kn(N/cm):  {kn!r}
Static_Friction:  {mu!r}
Kinetic_Friction: {mu!r}
Particle_Surface
COR:       {cor!r}
Kn(N/cm):  {kn!r}
Static_Friction:  {mu!r}
Kinetic_Friction: {mu!r}
Particle_Lifter
COR:       {cor!r}
Kn(N/cm):  {kn!r}
Static_Friction:  {mu!r}
Kinetic_Friction: {mu!r}
"""


def _orient(verts, faces, inside):
    """Order each face's vertices so the reference's face normal
    cross(V2, V1) (KSimulationData.cpp:846-856) points towards `inside(centroid)`."""
    out = []
    for f in faces:
        v = [np.asarray(verts[q], np.float64) for q in f]
        n = np.cross(v[2] - v[1], v[1] - v[0])
        c = np.mean(v, axis=0)
        if np.dot(n, np.asarray(inside(c), np.float64) - c) < 0:
            f = tuple(reversed(f))
        out.append(tuple(f))
    return out


def _write_wobj(path, title, verts, faces, tol=1.0):
    with open(path, "w") as fh:
        fh.write('Title: "%s"\nDescp: "synthetic"\nGeometry-Specfications\n' % title)
        fh.write("NUM_VERTEX: %d\n" % len(verts))
        for k, v in enumerate(verts):
            fh.write("%d %r %r %r\n" % (k + 1, float(v[0]), float(v[1]), float(v[2])))
        fh.write("NUM_SURFACES: %d\n" % len(faces))
        for k, f in enumerate(faces):
            fh.write('%d "F%d" Area_Tol: %r\nNUM_VERTEX: %d\n' % (k + 1, k, float(tol), len(f)))
            fh.write(" ".join(str(int(q) + 1) for q in f) + "\n")


def _write_cylinder_wobj(path, title, radius, height, offset, axis_normal=(0.0, 1.0, 0.0)):
    """Macro cylinder world object (KSimulationData.cpp:760-823): diameter,
    height, no caps, axis from the bottom-cap normal."""
    with open(path, "w") as fh:
        fh.write('Title: "%s"\nDescp: "synthetic"\nGeometry-Specfications\n' % title)
        fh.write("NUM_VERTEX: 0\nNUM_SURFACES: 1\n")
        fh.write('-1 "Cyl"\nDiameter: %r\nHeight: %r\nTop_Cap: false\nBot_Cap: false\n'
                 % (2.0 * radius, height))
        fh.write("Top_Normal: %r %r %r\n" % (-axis_normal[0], -axis_normal[1], -axis_normal[2]))
        fh.write("Bot_Normal: %r %r %r\n" % tuple(axis_normal))
        fh.write("Offset: %r %r %r\n" % tuple(offset))


def _write_project(root, name, world_name, *, title, sim_type, dt, wobjs, pobjs, counts, n, g,
                   rotation, roll_res, origin, world, cell, state, specific="", particle_type=0,
                   dobj_lines="Number: 0 Repeat: 0"):
    base = os.path.join(root, name)
    for sub in ("World", "SurfaceObjects", "ParticleObjects", "VolumeObjects"):
        os.makedirs(os.path.join(base, sub), exist_ok=True)
    wl = "\n".join("%d %s" % (k + 1, w) for k, w in enumerate(wobjs))
    pl = "\n".join("%d %s %d" % (k + 1, p, c) for k, (p, c) in enumerate(zip(pobjs, counts)))
    with open(os.path.join(base, "World", world_name + ".World"), "w") as fh:
        fh.write(_WORLD.format(title=title, sim_type=sim_type, ptype=particle_type, dt=dt,
                               n_w=len(wobjs), wobj_lines=wl,
                               n_p=len(pobjs), pobj_lines=pl, n=n, g=g, rotation=rotation,
                               roll_res=roll_res, origin=origin, world=world, cell=cell,
                               state=state, specific=specific, dobj_lines=dobj_lines))
    return base


_POBJ_POLY_PROPS = """------------------------
     2_POLY_PROP
------------------------
DENSITY:  {rho!r}
INERTIA_TENSOR:
1.0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
------------------------
     3_SPRING_DATA
------------------------
Particle_Particle
COR:       {cor!r}
Kn(N/cm):  {kn!r}
Friction:  {mu!r}
Friction:  {mu!r}
Particle_Surface
COR:       {cor!r}
Kn(N/cm):  {kn!r}
Friction:  {mu!r}
Friction:  {mu!r}
Particle_Lifter
COR:       {cor!r}
Kn(N/cm):  {kn!r}
Friction:  {mu!r}
Friction:  {mu!r}
"""


def dodecahedron(r):
    """Regular dodecahedron of circumradius r: 20 vertices, 12 pentagons
    (outward counter-clockwise), 30 edges."""
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(x, y, z) for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)]
    for a in (-1, 1):
        for b in (-1, 1):
            v += [(0, a / phi, b * phi), (a / phi, b * phi, 0), (b * phi, 0, a / phi)]
    v = np.array(v, np.float64)
    v *= r / np.linalg.norm(v[0])
    return _hull_polygons(v)


def cube(r):
    """Cube of circumradius r: 8 vertices, 6 squares, 12 edges."""
    h = r / math.sqrt(3.0)
    v = np.array([(x, y, z) for x in (-h, h) for y in (-h, h) for z in (-h, h)], np.float64)
    return _hull_polygons(v)


def hex_prism(r, aspect=1.0):
    """Hexagonal prism of circumradius r (height/width = aspect): 12
    vertices, 2 hexagons and 6 rectangles, 18 edges."""
    a = r / math.sqrt(1.0 + aspect * aspect)
    h = aspect * a
    v = [(a * math.cos(k * math.pi / 3), a * math.sin(k * math.pi / 3), z)
         for z in (-h, h) for k in range(6)]
    return _hull_polygons(np.array(v, np.float64))


def _hull_polygons(v):
    """Convex polyhedron from its vertices: faces as vertex lists ordered
    counter-clockwise seen from outside (merged coplanar hull triangles),
    and the edges."""
    from scipy.spatial import ConvexHull
    hull = ConvexHull(v)
    planes = {}
    for eq in hull.equations:
        key = tuple(np.round(eq, 6))
        planes[key] = eq
    faces = []
    for eq in planes.values():
        n, d = eq[:3], eq[3]
        idx = [i for i in range(len(v)) if abs(v[i] @ n + d) < 1e-9]
        c = v[idx].mean(axis=0)
        e1 = v[idx[0]] - c
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(n, e1)
        ang = [math.atan2((v[i] - c) @ e2, (v[i] - c) @ e1) for i in idx]
        faces.append([idx[i] for i in np.argsort(ang)])
    edges = set()
    for f in faces:
        for k in range(len(f)):
            a, b = f[k], f[(k + 1) % len(f)]
            edges.add((min(a, b), max(a, b)))
    return v, faces, sorted(edges)


def _write_pobj_poly(path, title, v, faces, edges, rho, kn, cor, mu):
    """A Format-0 polyhedral particle object (KSimulationData.cpp:1219-1624).
    The reference's parser takes a face normal from the face's vertices 3, 4
    and 1 (cross(V[2]-V[3], V[3]-V[0])), which points outwards for faces
    listed counter-clockwise seen from outside, as written here."""
    with open(path, "w") as fh:
        fh.write('Title: "%s"\nDescp: "synthetic"\nFormat(0=Man,1=Math): 0\n' % title)
        fh.write("------------------------\n1_Geometry_Specfications\n------------------------\n")
        fh.write("NUM_VERTEX: %d\n" % len(v))
        for k, p in enumerate(v):
            fh.write("%d %r %r %r\n" % (k + 1, float(p[0]), float(p[1]), float(p[2])))
        fh.write("NUM_FACES: %d\n" % len(faces))
        for k, f in enumerate(faces):
            fh.write("%d NUM_VERTEX: %d\n" % (k + 1, len(f)))
            fh.write(" ".join(str(q + 1) for q in f) + "\n")
        fh.write("NUM_EDGES: %d\n" % len(edges))
        for a, b in edges:
            fh.write("%d %d\n" % (a + 1, b + 1))
        fh.write(_POBJ_POLY_PROPS.format(rho=rho, kn=kn, cor=cor, mu=mu))


def random_quaternions(rng, n):
    """Uniformly distributed unit quaternions (w, x, y, z) with w >= 0."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1.0
    return q.astype(np.float32)


def poly_box_project(root, n=100_000, r=0.5, spacing=0.93, rho=2700.0, kn=1.0e5, cor=0.5,
                     mu=0.4, dt=1e-5, seed=2, name="PolyBox", world="Poly_box", jitter=0.02):
    """Convex polyhedra in a closed box: dodecahedra, cubes and hexagonal
    prisms of circumradius r (types 0, 1, 2 in turn) on a jittered cubic
    lattice of the given spacing, so that bounding spheres of lattice
    neighbours overlap and every particle starts with contacts (the first
    layer touches the three lower walls); random
    orientations, velocities N(0, 10 cm/s), spins N(0, 20 rad/s); y vertical;
    lattice positions jittered by U(-jitter, jitter) cm per coordinate.
    Returns (Project, state dict with a `quat` entry)."""
    base = os.path.join(root, name)
    for sub in ("SurfaceObjects", "ParticleObjects"):
        os.makedirs(os.path.join(base, sub), exist_ok=True)
    side = int(math.ceil(n ** (1.0 / 3.0)))
    L = side * spacing + 2.0 * r + 1.0
    verts = [(0, 0, 0), (L, 0, 0), (L, L, 0), (0, L, 0), (0, 0, L), (L, 0, L), (L, L, L), (0, L, L)]
    faces = [(0, 1, 2, 3), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0), (4, 7, 6, 5)]
    faces = _orient(verts, faces, lambda c: (0.5 * L, 0.5 * L, 0.5 * L))
    _write_wobj(os.path.join(base, "SurfaceObjects", "Box.WOBJ"), "Box", verts, faces)
    shapes = [("Dodeca", dodecahedron(r)), ("Cube", cube(r)), ("HexPrism", hex_prism(r))]
    for title, (v, f, e) in shapes:
        _write_pobj_poly(os.path.join(base, "ParticleObjects", title + ".POBJ"), title, v, f, e,
                         rho, kn, cor, mu)
    counts = [len(range(t, n, len(shapes))) for t in range(len(shapes))]
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij"),
                 axis=-1).reshape(-1, 3)[:n]
    # the first lattice layer 0.94 r from the three lower walls: vertices
    # that point at a wall touch it
    pos = (g * spacing + 0.94 * r + rng.uniform(-jitter, jitter, size=(n, 3)))
    # the parser's objects carry their centre of mass in the file frame
    # (here the origin up to rounding); positions are centres of mass
    ptype = np.arange(n, dtype=np.uint32) % len(shapes)
    order = np.argsort(ptype, kind="stable")
    state = dict(pos=pos[order].astype(np.float32),
                 vel=rng.normal(scale=10.0, size=(n, 3)).astype(np.float32),
                 avel=rng.normal(scale=20.0, size=(n, 3)).astype(np.float32),
                 quat=random_quaternions(rng, n), pid=np.arange(n, dtype=np.int32),
                 type=ptype[order])
    cell = 2.0 * r
    _write_project(root, name, world, title="Poly_box", sim_type=0, dt=dt, wobjs=["Box"],
                   pobjs=[t for t, _ in shapes], counts=counts, n=n, g=(0.0, -981.0, 0.0),
                   rotation=1, roll_res=0.0, origin=(-cell, -cell, -cell),
                   world=(L + cell, L + cell, L + cell), cell=cell, state="none",
                   particle_type=1)
    return Project.load(root, name, world), state


def box_project(root, n_side=(20, 20, 25), radius=0.1, rho=2500.0, box=10.0, kn=1.0e5, cor=0.5,
                mu=0.4, dt=1e-5, pitch=0.3, start=0.3, jitter=0.02, seed=0, cell=0.2,
                gravity=(0.0, 0.0, -981.0), name="Particles_Box", world="Box_plain"):
    """Particles_Box plain configuration: spheres on a jittered cubic lattice
    (x, y horizontal, z vertical) in a closed cube of six quad faces.
    Returns (Project, state dict)."""
    nx, ny, nz = n_side
    n = nx * ny * nz
    base = os.path.join(root, name)
    os.makedirs(os.path.join(base, "SurfaceObjects"), exist_ok=True)
    os.makedirs(os.path.join(base, "ParticleObjects"), exist_ok=True)
    L = float(box)
    verts = [(0, 0, 0), (L, 0, 0), (L, L, 0), (0, L, 0), (0, 0, L), (L, 0, L), (L, L, L), (0, L, L)]
    # quads ordered so cross(V2, V1) (KSimulationData.cpp:846-856) points into the box
    faces = [(0, 1, 2, 3), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0), (4, 7, 6, 5)]
    faces = _orient(verts, faces, lambda c: (0.5 * L, 0.5 * L, 0.5 * L))
    _write_wobj(os.path.join(base, "SurfaceObjects", "Box.WOBJ"), "Box", verts, faces)
    with open(os.path.join(base, "ParticleObjects", "Sphere.POBJ"), "w") as fh:
        fh.write(_POBJ.format(title="Sphere", diam=2.0 * radius, rho=rho, cor=cor, kn=kn, mu=mu))
    rng = np.random.default_rng(seed)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    lat = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1).astype(np.float64) * pitch + start
    pos = (lat + rng.uniform(-jitter, jitter, size=lat.shape)).astype(np.float32)
    state = dict(pos=pos, vel=np.zeros((n, 3), np.float32), avel=np.zeros((n, 3), np.float32),
                 pid=np.arange(n, dtype=np.int32), type=np.zeros(n, np.uint32))
    write_state_file(os.path.join(base, "Start_" + world), state)
    origin = (-cell, -cell, -cell)
    _write_project(root, name, world, title="Particles_Box", sim_type=0, dt=dt, wobjs=["Box"],
                   pobjs=["Sphere"], counts=[n], n=n, g=gravity, rotation=1, roll_res=0.0,
                   origin=origin, world=(L + cell, L + cell, L + cell), cell=cell,
                   state="Start_" + world)
    proj = Project.load(root, name, world)
    return proj, proj.read_state()


def cone_hopper_faces(r_top, r_out, y_top, y_out, n_seg):
    """Planar quads approximating a cone (axis +y, centred on x=z=r_top),
    n_seg segments around; each quad's normal points inward/upward."""
    quads = []
    c = r_top
    for k in range(n_seg):
        a0 = 2 * math.pi * k / n_seg
        a1 = 2 * math.pi * (k + 1) / n_seg
        p = [(c + r_top * math.cos(a0), y_top, c + r_top * math.sin(a0)),
             (c + r_top * math.cos(a1), y_top, c + r_top * math.sin(a1)),
             (c + r_out * math.cos(a1), y_out, c + r_out * math.sin(a1)),
             (c + r_out * math.cos(a0), y_out, c + r_out * math.sin(a0))]
        quads.append(p)
    return quads


def silo_project(root, n=1_000_000, r_min=0.2, r_max=0.4, n_bins=6, rho=2600.0, silo_r=25.0,
                 silo_h=100.0, half_angle_deg=30.0, outlet_d=6.0, seg_per_obj=4, n_sectors=7,
                 kn=1.0e5, cor=0.6, mu=0.5, dt=5e-6, seed=1, overlap=1e-5, rotation=0,
                 name="Silo", world="Silo_discharge", gravity=(0.0, -981.0, 0.0)):
    """Silo discharge, reference-law variant (y vertical, as the reference's
    silo logic assumes, main.cpp:271 and GPU_Memory_Transfer.cuh:656): a
    barrel of radius silo_r over a conical hopper of half-angle
    half_angle_deg down to an outlet of outlet_d, both faceted into
    n_sectors * seg_per_obj planar quads around, one world object per sector
    holding its hopper and barrel quads (the reference's limits: 8 world
    objects of at most 16 vertices and 16 faces), then the hatch.  Planar
    faces only, as the reference's own silo project (Projects/2.Silo: Tank,
    Container, Floor and Hatch objects): a macro cylinder would overwrite the
    forces of the hopper faces it meets at the junction (the reference's
    cylinder force replaces, DEM_Kernels_Compute.cuh:493), and the particles
    there sink through the hopper.  The barrel reaches 2 cm above the
    initial packing.  Radii uniform in [r_min, r_max] quantised to n_bins
    particle objects (the reference's 6-entry pair table).
    Rotation is off by default: the reference's tangential force scales with
    |v_t| / |v_rel| where v_t carries the spin term and v_rel does not
    (Collision_Response.cuh:430-466), which diverges for spinning particles
    in resting contact; the reference's own box world runs without rotation
    (Projects/1.Particles_Box/World/Spheres_128cm.World).
    Returns (Project, state dict)."""
    base = os.path.join(root, name)
    for sub in ("SurfaceObjects", "ParticleObjects"):
        os.makedirs(os.path.join(base, sub), exist_ok=True)
    r_out = 0.5 * outlet_d
    h_hop = (silo_r - r_out) / math.tan(math.radians(half_angle_deg))
    y_out = 10.0
    y_top = y_out + h_hop
    n_seg = seg_per_obj * n_sectors
    edges = np.linspace(r_min, r_max, n_bins + 1)
    radii = 0.5 * (edges[:-1] + edges[1:])
    rng = np.random.default_rng(seed)
    rs = rng.uniform(r_min, r_max, size=n)
    types = np.clip(np.searchsorted(edges, rs, side="right") - 1, 0, n_bins - 1).astype(np.uint32)
    counts = np.bincount(types, minlength=n_bins)
    pobjs = []
    for b in range(n_bins):
        nm = "Sphere%d" % b
        with open(os.path.join(base, "ParticleObjects", nm + ".POBJ"), "w") as fh:
            fh.write(_POBJ.format(title=nm, diam=float(2.0 * radii[b]), rho=float(rho), cor=float(cor), kn=float(kn), mu=float(mu)))
        pobjs.append(nm)
    # Size-banded simple-cubic layers: the particles of each radius bin fill
    # horizontal layers (largest bin lowest) on a lattice of pitch
    # 2 r (1 - overlap), so the bed starts as a contact network under load
    # (about six contacts per particle, solid fraction ~0.52) instead of a
    # free fall; each layer is clipped to the inscribed radius of the
    # faceted hopper (R cos(pi / segments)) / the barrel, with a clearance
    # of r / cos(half-angle) + 0.002 cm from the wall, so the bed rests on
    # the hopper almost at once.
    tan_a = math.tan(math.radians(half_angle_deg))
    cos_a = math.cos(math.radians(half_angle_deg))
    c = silo_r
    pos = np.zeros((n, 3), np.float64)
    types_out = np.zeros(n, np.uint32)
    k = 0
    y_last, r_last = None, None   # centre height and radius of the last layer laid
    for b in range(n_bins - 1, -1, -1):
        r = float(radii[b])
        pitch = 2.0 * r * (1.0 - overlap)
        need = int(counts[b])
        # the first layer of a bin rests on the last layer of the bin below
        # (the same relative overlap), so no bin starts in free fall
        y = y_out + 0.05 + r if y_last is None else y_last + (r_last + r) * (1.0 - overlap)
        while need > 0:
            # inscribed radius of the faceted hopper / barrel at this height,
            # less the sphere's reach to the wall (slanted in the hopper)
            inscribed = math.cos(math.pi / n_seg)
            if y < y_top:
                ra = (r_out + (y - y_out) * tan_a) * inscribed - (r / cos_a + 0.002)
            else:
                ra = silo_r * inscribed - (r + 0.002)
            if ra > 0:
                m = int(ra / pitch)
                g = np.arange(-m, m + 1) * pitch
                xx, zz = np.meshgrid(g, g, indexing="ij")
                keep = xx ** 2 + zz ** 2 <= ra * ra
                xs, zs = xx[keep][:need], zz[keep][:need]
                cnt = len(xs)
                pos[k:k + cnt, 0] = c + xs
                pos[k:k + cnt, 1] = y
                pos[k:k + cnt, 2] = c + zs
                types_out[k:k + cnt] = b
                k += cnt
                need -= cnt
                y_last = y
            y += pitch
        r_last = r
    types = types_out
    pos = pos.astype(np.float32)
    # world objects: per sector the hopper quads (outlet ring to hopper top)
    # and the barrel quads (hopper top to the barrel top), vertex rings
    # outlet / hopper top / barrel top
    y_bar = float(pos[:, 1].max()) + 2.0
    wobjs = []
    for o in range(n_sectors):
        vs, fs = [], []
        for k in range(seg_per_obj + 1):
            a = 2 * math.pi * (o * seg_per_obj + k) / n_seg
            ca, sa = math.cos(a), math.sin(a)
            vs += [(c + r_out * ca, y_out, c + r_out * sa), (c + silo_r * ca, y_top, c + silo_r * sa),
                   (c + silo_r * ca, y_bar, c + silo_r * sa)]
        for k in range(seg_per_obj):
            b0, b1 = 3 * k, 3 * (k + 1)
            fs.append((b0 + 1, b1 + 1, b1, b0))          # hopper quad
            fs.append((b0 + 2, b1 + 2, b1 + 1, b0 + 1))  # barrel quad
        nm = "Sector%d" % o
        # normals point into the silo: towards the axis (and up the cone)
        fs = _orient(vs, fs, lambda cc: (silo_r, cc[1] + 10.0, silo_r))
        _write_wobj(os.path.join(base, "SurfaceObjects", nm + ".WOBJ"), nm, vs, fs)
        wobjs.append(nm)
    # last world object: the hatch under the outlet (the removal height is
    # its first vertex's y - 5, main.cpp:771-773); opening it drops it
    yh = y_out - 1.0
    hv = [(silo_r - 2 * r_out, yh, silo_r - 2 * r_out), (silo_r + 2 * r_out, yh, silo_r - 2 * r_out),
          (silo_r + 2 * r_out, yh, silo_r + 2 * r_out), (silo_r - 2 * r_out, yh, silo_r + 2 * r_out)]
    _write_wobj(os.path.join(base, "SurfaceObjects", "Hatch.WOBJ"), "Hatch", hv,
                _orient(hv, [(0, 1, 2, 3)], lambda cc: (cc[0], cc[1] + 1.0, cc[2])))
    wobjs.append("Hatch")
    state = dict(pos=pos, vel=np.zeros((n, 3), np.float32), avel=np.zeros((n, 3), np.float32),
                 pid=np.arange(n, dtype=np.int32), type=types)
    write_state_file(os.path.join(base, "Start_" + world), state, sim_type=2)
    cell = 2.0 * r_max
    y_max = float(pos[:, 1].max()) + 4 * r_max
    origin = (-cell, -cell, -cell)
    worldsz = (2 * silo_r + cell, y_max, 2 * silo_r + cell)
    specific = ("_________________________________________________\n"
                "          6_Simulation_Specfic_Options\n"
                "Hatch_mode:        1\nFlow_counter:      1 1000\nkill_after:        1\n"
                "_________________________________________________\n")
    _write_project(root, name, world, title="Silo", sim_type=2, dt=dt, wobjs=wobjs, pobjs=pobjs,
                   counts=[int(c_) for c_ in counts], n=n, g=gravity, rotation=rotation, roll_res=0.0,
                   origin=origin, world=tuple(float(v) for v in worldsz), cell=float(cell), state="Start_" + world,
                   specific=specific)
    proj = Project.load(root, name, world)
    return proj, proj.read_state()


def mill_project(root, n=100_000, r_min=0.3, r_max=0.6, n_bins=6, rho=7800.0, drum_r=50.0,
                 drum_l=30.0, rpm=30.0, n_lifters=8, lifter_w=4.0, lifter_h=4.0, kn=1.0e6,
                 cor=0.4, mu=0.6, dt=2e-6, seed=2, overlap=1e-5, name="Mill", world="Mill_C3"):
    """Ball mill on the reference path: a drum of radius drum_r and length
    drum_l along z (macro cylinder with both end plates, centre line
    (drum_r, drum_r)), n_lifters box lifters of lifter_w x lifter_h along
    it (one lifter file, copied around the drum by the reference's Repeat,
    KSimulationData.cpp:1885-2028), mill speed rpm with power tallies on
    (Power(Revs) 1).  Spheres: radii uniform in [r_min, r_max] in n_bins
    particle objects, steel, linear law kn, e, mu; packed from the bottom of
    the drum on a simple-cubic lattice of pitch 2 r (1 - overlap), largest
    bin lowest, inside the circle the lifters leave free (drum_r - lifter_h
    - 1 cm), clear of the end plates.  The drum holds about 1.5e5 of these
    spheres at that lattice fill.  Returns (Project, state dict)."""
    base = os.path.join(root, name)
    for sub in ("SurfaceObjects", "ParticleObjects", "LifterObjects"):
        os.makedirs(os.path.join(base, sub), exist_ok=True)
    R, L = float(drum_r), float(drum_l)
    with open(os.path.join(base, "SurfaceObjects", "Drum.WOBJ"), "w") as fh:
        fh.write('Title: "DRUM_MILL"\nDescp: "synthetic"\nGeometry-Specfications\n'
                 "NUM_VERTEX: 0\nNUM_SURFACES: 1\n")
        fh.write('-1 "DRUM"\nDiameter: %r\nHeight: %r\nTop: true\nBot: true\n'
                 % (2.0 * R, L + 0.1))
        fh.write("normalT: 0.0 0.0 -1.0\nnormalB: 0.0 0.0 1.0\nOffset: 0.0 0.0 0.0\n")
    x0, x1 = R - 0.5 * lifter_w, R + 0.5 * lifter_w
    h = float(lifter_h)
    lv = [(x0, 0.0, 0.0), (x0, 0.0, L), (x1, 0.0, L), (x1, 0.0, 0.0),
          (x0, h, 0.0), (x0, h, L), (x1, h, L), (x1, h, 0.0)]
    with open(os.path.join(base, "LifterObjects", "Lifter.DOBJ"), "w") as fh:
        fh.write('Title: "Lifter"\nDescp: "Lifter"\nGeometry_Specfications: 1\n')
        fh.write("AXIS: 1.0 1.0 0.0\nCOM: %r %r %r\nB_R: %r\n" % (R, 0.5 * h, 0.5 * L,
                                                                  float(max(lifter_w, h))))
        fh.write("NUM_VERTEX: 8\n")
        for k, v in enumerate(lv):
            fh.write("%d %r %r %r\n" % (k + 1, v[0], v[1], v[2]))
        # the two side faces and the top, normals out of the lifter; the top's
        # two long edges
        fh.write('NUM_FACES: 3\n1 "Left" AreaTol: 0.10\nNUM_VERTEX: 4\n1 5 6 2\n'
                 '3 "Right" AreaTol: 0.10\nNUM_VERTEX: 4\n3 7 8 4\n'
                 '5 "Top" AreaTol: 0.10\nNUM_VERTEX: 4\n7 6 5 8\n'
                 "NUM_EDGES: 2\n5 6\n7 8\n")
    edges = np.linspace(r_min, r_max, n_bins + 1)
    radii = 0.5 * (edges[:-1] + edges[1:])
    rng = np.random.default_rng(seed)
    rs = rng.uniform(r_min, r_max, size=n)
    types = np.clip(np.searchsorted(edges, rs, side="right") - 1, 0, n_bins - 1).astype(np.uint32)
    counts = np.bincount(types, minlength=n_bins)
    pobjs = []
    for b in range(n_bins):
        nm = "Ball%d" % b
        with open(os.path.join(base, "ParticleObjects", nm + ".POBJ"), "w") as fh:
            fh.write(_POBJ.format(title=nm, diam=float(2.0 * radii[b]), rho=float(rho),
                                  cor=float(cor), kn=float(kn), mu=float(mu)))
        pobjs.append(nm)
    r_in = R - h - 1.0
    pos = np.zeros((n, 3), np.float64)
    types_out = np.zeros(n, np.uint32)
    k = 0
    y = R - r_in
    for b in range(n_bins - 1, -1, -1):
        r = float(radii[b])
        pitch = 2.0 * r * (1.0 - overlap)
        need = int(counts[b])
        y += r
        zs_all = np.arange(r + 0.05, L - r - 0.05 + 1e-9, pitch)
        while need > 0:
            if y > R + r_in - r:
                raise ValueError("mill_project: %d spheres do not fit the drum" % n)
            half = math.sqrt(max(r_in * r_in - (y - R) ** 2, 0.0)) - r - 0.002
            if half > 0:
                m = int(half / pitch)
                xs = R + np.arange(-m, m + 1) * pitch
                xx, zz = np.meshgrid(xs, zs_all, indexing="ij")
                xx, zz = xx.ravel()[:need], zz.ravel()[:need]
                cnt = len(xx)
                pos[k:k + cnt, 0] = xx
                pos[k:k + cnt, 1] = y
                pos[k:k + cnt, 2] = zz
                types_out[k:k + cnt] = b
                k += cnt
                need -= cnt
            y += pitch
        y += r * 0.002
    state = dict(pos=pos.astype(np.float32), vel=np.zeros((n, 3), np.float32),
                 avel=np.zeros((n, 3), np.float32), pid=np.arange(n, dtype=np.int32),
                 type=types_out)
    write_state_file(os.path.join(base, "Start_" + world), state, sim_type=1)
    cell = 2.0 * r_max
    origin = (-cell, -cell, -cell)
    worldsz = (2 * R + 2 * cell, 2 * R + 2 * cell, L + 2 * cell)
    specific = ("_________________________________________________\n"
                "          6_Simulation_Specfic_Options\n"
                "Power(Revs):   1\nTotal(Revs):   5\nSpeed(RPM):    %r\n"
                "_________________________________________________\n" % float(rpm))
    _write_project(root, name, world, title="Mill", sim_type=1, dt=dt, wobjs=["Drum"],
                   pobjs=pobjs, counts=[int(c_) for c_ in counts], n=n, g=(0.0, -981.0, 0.0),
                   rotation=1, roll_res=0.0, origin=origin,
                   world=tuple(float(v) for v in worldsz), cell=float(cell),
                   state="Start_" + world, specific=specific,
                   dobj_lines="Number: 1 Repeat: %d\n1 Lifter" % n_lifters)
    proj = Project.load(root, name, world)
    return proj, proj.read_state()


# ---------------------------------------------------------------- ensembles
def lattice_fill(n, lo, hi, pitch, rng, jitter=0.0):
    """First n sites of a face-centred cubic lattice of nearest-neighbour
    distance `pitch` inside the box [lo, hi] (filled bottom up, z last; n
    None: all of them), each moved by a uniform jitter in [-jitter, jitter]."""
    a = pitch * math.sqrt(2.0)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    m = np.floor((hi - lo) / a).astype(int) + 1
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    pts = []
    for iz in range(m[2]):
        layer = []
        for iy in range(m[1]):
            for ix in range(m[0]):
                layer.append(base + lo + np.array([ix, iy, iz]) * a)
        layer = np.concatenate(layer)
        layer = layer[np.all((layer >= lo) & (layer <= hi), axis=1)]
        pts.append(layer[np.lexsort((layer[:, 0], layer[:, 1], layer[:, 2]))])
        if n is not None and sum(len(p) for p in pts) >= n:
            break
    pts = np.concatenate(pts)
    if n is None:
        n = len(pts)
    if len(pts) < n:
        raise ValueError("box holds %d lattice sites, %d requested" % (len(pts), n))
    pts = pts[:n]
    if jitter > 0:
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    return pts


def box_walls(L, H, z0=0.0):
    """Six inward planes of the box [0, L] x [0, L] x [z0, z0 + H]."""
    from . import ensemble as E
    return [E.plane((1, 0, 0), 0.0), E.plane((-1, 0, 0), -L), E.plane((0, 1, 0), 0.0),
            E.plane((0, -1, 0), -L), E.plane((0, 0, 1), z0), E.plane((0, 0, -1), -(z0 + H))]


def box_system(n, L, H, cell, wall0, *, density, kn=1e5, kt_ratio=2.0 / 7.0, youngs=0.0,
               poisson=0.3, restitution=0.5, mu=0.4, mu_wall=None, mu_roll=0.0,
               gravity=(0.0, 0.0, -981.0)):
    """A blaze_system for a box [0, L]^2 x [0, H] whose six planes are
    walls[wall0 .. wall0 + 6)."""
    from . import ensemble as E
    s = E.System()
    s.n = int(n)
    margin = 0.5 * cell
    for k in range(3):
        s.origin[k] = -margin
    s.cell = cell
    ext = (L, L, H)
    for k in range(3):
        s.ncells[k] = int(math.ceil((ext[k] + 2 * margin) / cell))
    for k in range(3):
        s.gravity[k] = gravity[k]
    s.density = density
    s.kn, s.kt_ratio, s.youngs, s.poisson = kn, kt_ratio, youngs, poisson
    s.restitution, s.mu = restitution, mu
    s.mu_wall = mu if mu_wall is None else mu_wall
    s.mu_roll = mu_roll
    s.wall0, s.nwalls, s.tri0, s.ntris = wall0, 6, 0, 0
    return s


def box_ensemble(counts, *, r_min=0.1, r_max=0.2, solid_fraction=0.55, height_factor=3.0,
                 rho=2500.0, kn=1e5, kt_ratio=2.0 / 7.0, mus=None, restitutions=None,
                 skin=0.02, seed=3, gravity=(0.0, 0.0, -981.0)):
    """Independent box-settling systems: system s holds counts[s] spheres with
    radii uniform in [r_min, r_max] (cm), in a box of square base L_s with
    L_s^3 = (total sphere volume) / solid_fraction and height
    height_factor * L_s (room for the loose initial lattice above the settled
    bed); spheres start on an FCC lattice of nearest-neighbour distance
    2 r_max + skin / 2, jittered by at most a fifth of the lattice gap, at rest.  Per-system friction
    and restitution from `mus` / `restitutions`.  Returns (systems, walls,
    pos, radius) with the arrays concatenated in system order."""
    rng = np.random.default_rng(seed)
    density = rho * 1e-6  # kg/cm^3
    cell = 2.0 * r_max + skin
    systems, walls, pos, rad = [], [], [], []
    for s, n in enumerate(counts):
        r = rng.uniform(r_min, r_max, size=int(n))
        vol = float(np.sum(4.0 / 3.0 * math.pi * r ** 3))
        L = (vol / solid_fraction) ** (1.0 / 3.0)
        H = height_factor * L
        pitch = 2.0 * r_max + 0.5 * skin
        # jitter small enough that no two lattice neighbours start in contact
        jitter = min(0.1 * r_min, 0.2 * (pitch - 2.0 * r_max))
        p = lattice_fill(int(n), (r_max + 0.01, r_max + 0.01, r_max + 0.01),
                         (L - r_max - 0.01, L - r_max - 0.01, H - r_max - 0.01), pitch, rng,
                         jitter=jitter)
        mu = 0.4 if mus is None else float(mus[s])
        e = 0.5 if restitutions is None else float(restitutions[s])
        systems.append(box_system(n, L, H, cell, len(walls), density=density, kn=kn,
                                  kt_ratio=kt_ratio, restitution=e, mu=mu, gravity=gravity))
        walls += box_walls(L, H)
        pos.append(p.astype(np.float32))
        rad.append(r.astype(np.float32))
    return systems, walls, np.concatenate(pos), np.concatenate(rad)


def box_system_project(root, name, system, L, H, radii, rho, dt=1e-5):
    """The reference project of one box system of an ensemble: the box
    [0, L]^2 x [0, H] as six quads, one particle object per distinct radius
    in `radii` (diameter 2 r, density rho kg/m^3, the system's kn,
    restitution and friction for pairs, surfaces and lifters), the system's
    cell size and gravity (as many cells on every axis as the longest one
    needs), rotation on.  With BLAZE_LAW_REFERENCE the ensemble
    steps the same system with the same laws.  Returns (Project, types),
    types[k] the particle object of radius radii[k]."""
    base = os.path.join(root, name)
    for sub in ("SurfaceObjects", "ParticleObjects"):
        os.makedirs(os.path.join(base, sub), exist_ok=True)
    L, H = float(L), float(H)
    verts = [(0, 0, 0), (L, 0, 0), (L, L, 0), (0, L, 0), (0, 0, H), (L, 0, H), (L, L, H), (0, L, H)]
    faces = [(0, 1, 2, 3), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0), (4, 7, 6, 5)]
    faces = _orient(verts, faces, lambda c: (0.5 * L, 0.5 * L, 0.5 * H))
    _write_wobj(os.path.join(base, "SurfaceObjects", "Box.WOBJ"), "Box", verts, faces)
    rs = np.asarray(radii, np.float32)
    bins = np.unique(rs)
    types = np.searchsorted(bins, rs).astype(np.uint32)
    pobjs = []
    f32 = lambda v: float(np.float32(v))  # noqa: E731  (the ensemble's float values)
    for b, r in enumerate(bins):
        nm = "Ball%d" % b
        with open(os.path.join(base, "ParticleObjects", nm + ".POBJ"), "w") as fh:
            fh.write(_POBJ.format(title=nm, diam=2.0 * float(r), rho=float(rho),
                                  cor=f32(system.restitution), kn=f32(system.kn),
                                  mu=f32(system.mu)))
        pobjs.append(nm)
    counts = [int(c) for c in np.bincount(types, minlength=len(bins))]
    cell = f32(system.cell)
    origin = tuple(f32(system.origin[k]) for k in range(3))
    # the same cell count on every axis: the reference's hash
    # x + z nz + y nx nz (BroadPhase.cuh:42-50) indexes past its cell table
    # when nx < nz, and the grid only has to cover the box
    nc = max(int(system.ncells[k]) for k in range(3))
    world = tuple(float(np.float32(origin[k] + nc * cell)) for k in range(3))
    _write_project(root, name, "Box", title=name, sim_type=0, dt=dt, wobjs=["Box"], pobjs=pobjs,
                   counts=counts, n=len(rs), g=tuple(f32(system.gravity[k]) for k in range(3)),
                   rotation=1, roll_res=f32(system.mu_roll), origin=origin, world=world,
                   cell=cell, state="none")
    return Project.load(root, name, "Box"), types


def cone_hopper_triangles(silo_r, r_out, y_top, y_out, n_seg=64, n_ring=32, centre=None):
    """A cone (axis +y) from radius r_out at y_out to silo_r at y_top as
    n_seg x n_ring quads, each split into two triangles (2 n_seg n_ring
    triangles), vertices on the cone."""
    c = silo_r if centre is None else centre
    tris = []
    for k in range(n_ring):
        y0 = y_out + (y_top - y_out) * k / n_ring
        y1 = y_out + (y_top - y_out) * (k + 1) / n_ring
        r0 = r_out + (silo_r - r_out) * k / n_ring
        r1 = r_out + (silo_r - r_out) * (k + 1) / n_ring
        for m in range(n_seg):
            a0 = 2 * math.pi * m / n_seg
            a1 = 2 * math.pi * (m + 1) / n_seg
            p00 = (c + r0 * math.cos(a0), y0, c + r0 * math.sin(a0))
            p01 = (c + r0 * math.cos(a1), y0, c + r0 * math.sin(a1))
            p10 = (c + r1 * math.cos(a0), y1, c + r1 * math.sin(a0))
            p11 = (c + r1 * math.cos(a1), y1, c + r1 * math.sin(a1))
            tris.append((p00, p01, p11))
            tris.append((p00, p11, p10))
    return tris


def drum_mesh_triangles(R, L, n_seg, n_len, n_lifters=8, lifter_w=4.0, lifter_h=4.0,
                        end_fans=True):
    """A ball-mill drum as triangles: the barrel (radius R, axis z, from z = 0
    to L) as n_seg x n_len quads, the two end plates as fans of n_seg
    triangles about the axis (end_fans), and n_lifters box lifters
    (lifter_w wide, lifter_h high, the drum's length) on the barrel, each as
    its two sides and top, each face split along its length into n_len
    quads; every quad is two triangles.  The axis passes through (0, 0).
    Returns a list of triangles ((x, y, z) x 3)."""
    tris = []
    zs = np.linspace(0.0, L, n_len + 1)
    for m in range(n_seg):
        a0, a1 = 2 * math.pi * m / n_seg, 2 * math.pi * (m + 1) / n_seg
        for k in range(n_len):
            p00 = (R * math.cos(a0), R * math.sin(a0), zs[k])
            p01 = (R * math.cos(a1), R * math.sin(a1), zs[k])
            p10 = (R * math.cos(a0), R * math.sin(a0), zs[k + 1])
            p11 = (R * math.cos(a1), R * math.sin(a1), zs[k + 1])
            tris += [(p00, p01, p11), (p00, p11, p10)]
        for z in ((0.0, L) if end_fans else ()):
            tris.append(((0.0, 0.0, z), (R * math.cos(a0), R * math.sin(a0), z),
                         (R * math.cos(a1), R * math.sin(a1), z)))
    for q in range(n_lifters):
        ang = 2 * math.pi * q / n_lifters
        er = np.array([math.cos(ang), math.sin(ang), 0.0])    # outward
        et = np.array([-math.sin(ang), math.cos(ang), 0.0])   # along the barrel
        # the lifter's foot sits on the chord at R cos(half angle) so its
        # corners touch the barrel
        half = 0.5 * lifter_w
        base = math.sqrt(R * R - half * half)
        top = base - lifter_h
        corners = {"bl": base * er - half * et, "br": base * er + half * et,
                   "tl": top * er - half * et, "tr": top * er + half * et}
        faces = [("bl", "tl"), ("tl", "tr"), ("tr", "br")]   # side, top, side
        for u, v in faces:
            for k in range(n_len):
                a = tuple(corners[u][:2]) + (zs[k],)
                b = tuple(corners[v][:2]) + (zs[k],)
                c = tuple(corners[v][:2]) + (zs[k + 1],)
                d = tuple(corners[u][:2]) + (zs[k + 1],)
                tris += [(a, b, c), (a, c, d)]
    return tris


def drum_mesh_ensemble(n=100_000, R=50.0, L=30.0, n_seg=232, n_len=32, n_lifters=8,
                       lifter_w=4.0, lifter_h=4.0, r_min=0.3, r_max=0.6, rho=7800.0, kn=1e6,
                       restitution=0.4, mu=0.6, rpm=30.0, law_youngs=0.0, skin=0.04, seed=2,
                       gravity=(0.0, -981.0, 0.0)):
    """The ball mill with its drum and lifters as a turning triangle mesh
    (drum_mesh_triangles: 232 x 32 barrel quads and 8 lifters of 3 faces x
    32 quads, 16,384 triangles; the end plates are planes turning in place)
    as a one-system ensemble turning at rpm about the z axis: n spheres r ~ U[r_min, r_max]
    on a lattice in the lower part of the drum inside the lifter ring, at
    rest; linear law kn (kt = 2/7 kn), restitution, mu; y vertical.
    Returns (systems, walls, pos, radius)."""
    from . import ensemble as E
    tris = drum_mesh_triangles(R, L, n_seg, n_len, n_lifters, lifter_w, lifter_h, end_fans=False)
    walls = [E.plane((0, 0, 1), 0.0), E.plane((0, 0, -1), -L)] + [E.triangle(*t) for t in tris]
    s = E.System()
    s.n = int(n)
    cell = 2.0 * r_max + skin
    for k, (o, ext) in enumerate(zip((-R - cell, -R - cell, -cell),
                                     (2 * R + 2 * cell, 2 * R + 2 * cell, L + 2 * cell))):
        s.origin[k] = o
        s.ncells[k] = int(math.ceil(ext / cell))
    s.cell = cell
    for k in range(3):
        s.gravity[k] = gravity[k]
    s.density = rho * 1e-6
    s.kn, s.kt_ratio, s.youngs, s.poisson = kn, 2.0 / 7.0, law_youngs, 0.3
    s.restitution, s.mu, s.mu_wall, s.mu_roll = restitution, mu, mu, 0.0
    s.wall0, s.nwalls, s.tri0, s.ntris = 0, 2, 2, len(tris)
    s.rot_axis[2] = 1.0
    s.rot_omega = -rpm * 2.0 * math.pi / 60.0
    rng = np.random.default_rng(seed)
    r_in = R - lifter_h - 1.0
    pitch = 2.0 * r_max + 0.5 * skin
    pts = lattice_fill(None, (-r_in, -r_in, r_max + 0.05), (r_in, r_in, L - r_max - 0.05),
                       pitch, rng, jitter=0.1 * (pitch - 2.0 * r_max))
    pts = pts[np.hypot(pts[:, 0], pts[:, 1]) < r_in - r_max]
    pts = pts[np.argsort(pts[:, 1], kind="stable")][:n]   # lowest first
    if len(pts) < n:
        raise ValueError("drum_mesh_ensemble: %d spheres do not fit the drum" % n)
    rad = rng.uniform(r_min, r_max, n)
    return [s], walls, pts.astype(np.float32), rad.astype(np.float32)


def silo_full_ensemble(n=1_000_000, r_min=0.2, r_max=0.4, rho=2600.0, silo_r=25.0,
                       silo_h=100.0, half_angle_deg=30.0, outlet_d=6.0, n_seg=64, n_ring=32,
                       youngs_pa=1e7, poisson=0.3, restitution=0.6, mu=0.5, mu_roll=0.01,
                       skin=0.04, seed=1, overlap=1e-5, gravity=(0.0, -981.0, 0.0)):
    """Silo discharge, full variant, as a one-system ensemble: 1,000,000
    spheres with radii uniform in [0.2, 0.4] cm (seed 1), density 2600
    kg/m^3, in a cylinder r = 25 cm, h = 100 cm over a 30 degree conical
    hopper of 2 x 64 x 32 = 4,096 triangles to a 6 cm outlet (open), a floor
    30 cm below the outlet to catch the discharge; Hertz-Mindlin with
    E = 1e7 Pa, nu = 0.3, restitution 0.6, mu = 0.5, rolling mu = 0.01; y
    vertical.  The spheres start in 24 size bands of horizontal layers on a
    lattice of pitch 2 r_band (1 - overlap) (largest band lowest, r_band the
    band's largest radius), clipped to the hopper's inscribed radius and the
    barrel with a small clearance, at rest: a contact network under load
    from the first step.  The layers are looser than a poured bed, so the
    column reaches above the 100 cm barrel (the silo has no lid; the grid
    covers it).  Returns (systems, walls, pos, radius)."""
    from . import ensemble as E
    rng = np.random.default_rng(seed)
    r = rng.uniform(r_min, r_max, size=n)
    r_out = 0.5 * outlet_d
    tan_a = math.tan(math.radians(half_angle_deg))
    cos_a = math.cos(math.radians(half_angle_deg))
    h_hop = (silo_r - r_out) / tan_a
    y_floor = 0.0
    y_out = y_floor + 30.0
    y_top = y_out + h_hop
    c = silo_r
    # layers by radius band, largest band lowest; the pitch of a band is set
    # by its largest radius
    order = np.argsort(-r, kind="stable")
    r = r[order]
    bands = np.array_split(np.arange(n), 24)
    pos = np.zeros((n, 3), np.float64)
    k = 0
    y = y_out + 0.05
    inscribed = math.cos(math.pi / n_seg)
    for idx in bands:
        rb = float(r[idx[0]])
        pitch = 2.0 * rb * (1.0 - overlap)
        need = len(idx)
        y += rb
        while need > 0:
            ra = (r_out + (y - y_out) * tan_a) * inscribed if y < y_top else silo_r
            ra -= rb / cos_a + 0.002
            if ra > 0:
                m = int(ra / pitch)
                g = np.arange(-m, m + 1) * pitch
                xx, zz = np.meshgrid(g, g, indexing="ij")
                keep = xx ** 2 + zz ** 2 <= ra * ra
                xs, zs = xx[keep][:need], zz[keep][:need]
                cnt = len(xs)
                pos[k:k + cnt, 0] = c + xs
                pos[k:k + cnt, 1] = y
                pos[k:k + cnt, 2] = c + zs
                k += cnt
                need -= cnt
            y += pitch
        y += rb * 0.002
    # the silo has no lid: a packing taller than the barrel (the simple-cubic
    # layers are looser than a poured bed) continues above it
    y_max = max(float(pos[:, 1].max()) + 2.0 * r_max, y_top + silo_h)
    walls = [E.cylinder((c, 0.0, c), (0.0, 1.0, 0.0), silo_r), E.plane((0.0, 1.0, 0.0), y_floor)]
    tri = cone_hopper_triangles(silo_r, r_out, y_top, y_out, n_seg, n_ring)
    walls += [E.triangle(*t) for t in tri]
    cell = 2.0 * r_max + skin
    s = E.System()
    s.n = int(n)
    origin = (-cell, y_floor - cell, -cell)
    ext = (2.0 * silo_r + 2.0 * cell, y_max - y_floor + 2.0 * cell, 2.0 * silo_r + 2.0 * cell)
    for q in range(3):
        s.origin[q] = origin[q]
        s.ncells[q] = int(math.ceil(ext[q] / cell))
        s.gravity[q] = gravity[q]
    s.cell = cell
    s.density = rho * 1e-6
    s.kn, s.kt_ratio = 0.0, 2.0 / 7.0
    s.youngs = youngs_pa * 0.01  # kg/(cm s^2)
    s.poisson = poisson
    s.restitution, s.mu, s.mu_wall, s.mu_roll = restitution, mu, mu, mu_roll
    s.wall0, s.nwalls, s.tri0, s.ntris = 0, 2, 2, len(tri)
    return [s], walls, pos.astype(np.float32), r.astype(np.float32)


def batched_counts(nsys=512, n_min=2000, n_max=50000, seed=3):
    """Particle counts log-uniform in [n_min, n_max] (the batched workload)."""
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=nsys))).astype(int)


def box_c1(n_side=(20, 20, 25), radius=0.1, rho=2500.0, box=10.0, kn=1.0e5, cor=0.5, mu=0.4,
           kt_ratio=2.0 / 7.0, pitch=0.3, start=0.3, jitter=0.02, seed=0, skin=0.02):
    """The Particles_Box configuration with the tangential history law, as a
    one-system ensemble: n_side spheres on a cubic lattice of pitch `pitch`
    from `start` (x, y horizontal, z vertical), each jittered uniformly by
    +-jitter (seed 0), at rest, in the cube [0, box]^3 of six planes; linear
    spring-dashpot kn, restitution cor, Coulomb mu, kt = kt_ratio kn, gravity
    -981 cm/s^2 along z.  Returns (systems, walls, pos, radius)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = n_side
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    lat = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1).astype(np.float64) * pitch + start
    pos = (lat + rng.uniform(-jitter, jitter, size=lat.shape)).astype(np.float32)
    n = len(pos)
    cell = 2.0 * radius + skin
    S = box_system(n, box, box, cell, 0, density=rho * 1e-6, kn=kn, kt_ratio=kt_ratio,
                   restitution=cor, mu=mu)
    return [S], box_walls(box, box), pos, np.full(n, radius, np.float32)


# ------------------------------------------------------- mixed charges
def hull_mass_centre(v, f):
    """Volume and centre of mass of the closed outward triangle mesh (v, f),
    FP64 (tetrahedra of the faces with the origin)."""
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    det = np.einsum("ij,ij->i", a, np.cross(b, c))
    vol = det.sum() / 6.0
    return vol, (det[:, None] * (a + b + c)).sum(axis=0) / 24.0 / vol


def rock_hull(rng, n_min=8, n_max=16, r_min=0.5, r_max=1.0):
    """A rock: the convex hull of n ~ U{n_min .. n_max} points uniform on a
    sphere of radius R ~ U[r_min, r_max] (cm), moved so that its centre of
    mass is the origin.  Returns (vertices (n, 3) float32, outward triangles
    (2 n - 4, 3) int32)."""
    from scipy.spatial import ConvexHull
    while True:
        n = int(rng.integers(n_min, n_max + 1))
        R = float(rng.uniform(r_min, r_max))
        p = rng.normal(size=(n, 3))
        p = p / np.linalg.norm(p, axis=1, keepdims=True) * R
        h = ConvexHull(p)
        if len(h.vertices) != n or len(h.simplices) != 2 * n - 4:
            continue
        f = h.simplices.copy()
        cen = p.mean(axis=0)
        for k in range(len(f)):
            a, b, c = p[f[k]]
            if np.dot(np.cross(b - a, c - a), a - cen) < 0:
                f[k] = f[k][[0, 2, 1]]
        _, com = hull_mass_centre(p, f)
        return (p - com).astype(np.float32), f.astype(np.int32)


def rock_shapes(n, seed=2, n_pts=(8, 16), radius=(0.5, 1.0), rho=2700.0):
    """n distinct rocks (rock_hull, seed) as ensemble Shapes of density rho
    (kg/m^3)."""
    from . import ensemble as E
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        v, f = rock_hull(rng, n_pts[0], n_pts[1], radius[0], radius[1])
        out.append(E.shape(v, f, rho * 1e-6))
    return out


def _mixed_placement(rng, sphere_sites, rock_sites, n_spheres, n_rocks, r_min, r_max, rock_rb,
                     height_axis, gap=0.02):
    """Rocks at n_rocks random sites of the rock lattice below a level h
    (rock k gets bounding radius rock_rb[k]), spheres (radii drawn per
    sphere site, U[r_min, r_max]) at the lowest n_spheres sites below h whose
    sphere keeps `gap` from every rock's bounding sphere: the lowest level
    (in steps of 0.5 cm) where both fit.  Returns (sphere centres, their
    radii, rock centres)."""
    from scipy.spatial import cKDTree
    rs = rng.uniform(r_min, r_max, len(sphere_sites))
    ys = sphere_sites[:, height_axis]
    yr = rock_sites[:, height_axis]
    rb = np.asarray(rock_rb, np.float64)
    reach = r_max + (rb.max() if len(rb) else 0.0) + gap
    h = min(ys.min(), yr.min())
    top = max(ys.max(), yr.max()) + 1.0
    while h <= top:
        cand = np.nonzero(yr < h)[0]
        if len(cand) >= n_rocks:
            sub = np.random.default_rng(int(rng.integers(1 << 31)))
            pick = np.sort(sub.choice(cand, n_rocks, replace=False))
            rocks = rock_sites[pick]
            ok = ys < h
            if n_rocks:
                kq = min(16, n_rocks)
                d, k = cKDTree(rocks).query(sphere_sites, k=kq, distance_upper_bound=reach)
                d, k = d.reshape(len(rs), kq), k.reshape(len(rs), kq)
                hit = k < n_rocks
                lim = rs[:, None] + rb[np.minimum(k, n_rocks - 1)] + gap
                ok &= ~np.any(hit & (d <= lim), axis=1)
            idx = np.nonzero(ok)[0]
            if len(idx) >= n_spheres:
                idx = idx[np.argsort(ys[idx], kind="stable")][:n_spheres]
                return sphere_sites[idx], rs[idx], rocks
        h += 0.5
    raise ValueError("the charge of %d spheres and %d rocks does not fit" % (n_spheres, n_rocks))


def _bounding_radius(s):
    return float(np.linalg.norm(np.asarray(s.verts).reshape(-1, 3)[:s.nverts], axis=1).max())


def mixed_charge_state(sph, sph_r, rocks, shapes, rng):
    """Caller arrays of a mixed charge: spheres first, then rocks (shape k
    for rock k, random orientations).  Returns (pos, radius, shape_of, quat)."""
    ns, nr = len(sph), len(rocks)
    pos = np.concatenate([sph, rocks]).astype(np.float32)
    rad = np.concatenate([sph_r, [_bounding_radius(s) for s in shapes[:nr]]])
    shape_of = np.concatenate([np.full(ns, -1), np.arange(nr)]).astype(np.int32)
    quat = np.zeros((ns + nr, 4), np.float32)
    quat[:ns, 0] = 1.0
    quat[ns:] = random_quaternions(rng, nr)
    return pos, rad.astype(np.float32), shape_of, quat


def mixed_box_ensemble(n_spheres=300, n_rocks=24, L=10.0, H=20.0, r_min=0.3, r_max=0.6,
                       rock_radius=(0.5, 1.0), rho=7800.0, rock_rho=2700.0, kn=1e6,
                       restitution=0.4, mu=0.6, skin=0.04, seed=2, gravity=(0.0, 0.0, -981.0)):
    """Steel balls and rocks in a closed box [0, L]^2 x [0, H] (six planes):
    rocks (rock_shapes, seed) at random sites of a lattice of pitch
    2 r_bound + 0.05 (r_bound the largest rock's bounding radius),
    balls r ~ U[r_min, r_max] on a lattice of pitch 2 r_max + skin / 2 clear
    of the rocks, at rest; linear law kn (kt = 2/7 kn), restitution, mu.
    Returns (systems, walls, pos, radius, shapes, shape_of, quat)."""
    rng = np.random.default_rng(seed)
    shapes = rock_shapes(n_rocks, seed=seed, radius=rock_radius, rho=rock_rho)
    rbs = [_bounding_radius(x) for x in shapes]
    rb = max([0.0] + rbs)
    cell = 2.0 * max(r_max, rb) + skin + 1e-3
    walls = box_walls(L, H)
    s = box_system(n_spheres + n_rocks, L, H, cell, 0, density=rho * 1e-6, kn=kn,
                   restitution=restitution, mu=mu, gravity=gravity)
    m = 0.05
    sph = lattice_fill(None, (r_max + m,) * 2 + (r_max + m,), (L - r_max - m,) * 2 + (H - r_max - m,),
                       2.0 * r_max + 0.5 * skin, rng)
    rk = lattice_fill(None, (rb + m,) * 2 + (rb + m,), (L - rb - m,) * 2 + (H - rb - m,),
                      2.0 * rb + 0.05, rng)
    sph, sph_r, rocks = _mixed_placement(rng, sph, rk, n_spheres, n_rocks, r_min, r_max, rbs, 2)
    pos, rad, shape_of, quat = mixed_charge_state(sph, sph_r, rocks, shapes, rng)
    return [s], walls, pos, rad, shapes, shape_of, quat


def mill_mixed_ensemble(n_spheres=100_000, n_rocks=5_000, R=50.0, L=30.0, n_seg=232, n_len=32,
                        n_lifters=8, lifter_w=4.0, lifter_h=4.0, r_min=0.3, r_max=0.6,
                        rho=7800.0, rock_radius=(0.5, 1.0), rock_rho=2700.0, kn=1e6,
                        restitution=0.4, mu=0.6, rpm=30.0, skin=0.04, seed=2,
                        gravity=(0.0, -981.0, 0.0)):
    """The ball mill's mixed charge: the drum and lifters as a turning mesh
    (drum_mesh_triangles, end plates as planes turning in place) with steel
    balls r ~ U[r_min, r_max] (density rho) and rocks (rock_shapes: hulls of
    8-16 points on spheres of radius rock_radius, seed, density rock_rho),
    the count ratio of the configuration's 2,000,000 : 100,000; rocks at
    random sites of a lattice of pitch 2 r_bound + 0.05 (r_bound the largest
    rock's bounding radius), balls on a lattice of
    pitch 2 r_max + skin / 2 clear of them, inside the lifter ring from the
    bottom up, at rest; linear law kn (kt = 2/7 kn), restitution, mu, rpm
    about z.  Returns (systems, walls, pos, radius, shapes, shape_of, quat)."""
    from . import ensemble as E
    rng = np.random.default_rng(seed)
    shapes = rock_shapes(n_rocks, seed=seed, radius=rock_radius, rho=rock_rho)
    rbs = [_bounding_radius(x) for x in shapes]
    rb = max([0.0] + rbs)
    tris = drum_mesh_triangles(R, L, n_seg, n_len, n_lifters, lifter_w, lifter_h, end_fans=False)
    walls = [E.plane((0, 0, 1), 0.0), E.plane((0, 0, -1), -L)] + [E.triangle(*t) for t in tris]
    s = E.System()
    s.n = int(n_spheres + n_rocks)
    cell = 2.0 * max(r_max, rb) + skin + 1e-3
    for k, (o, ext) in enumerate(zip((-R - cell, -R - cell, -cell),
                                     (2 * R + 2 * cell, 2 * R + 2 * cell, L + 2 * cell))):
        s.origin[k] = o
        s.ncells[k] = int(math.ceil(ext / cell))
    s.cell = cell
    for k in range(3):
        s.gravity[k] = gravity[k]
    s.density = rho * 1e-6
    s.kn, s.kt_ratio, s.youngs, s.poisson = kn, 2.0 / 7.0, 0.0, 0.3
    s.restitution, s.mu, s.mu_wall, s.mu_roll = restitution, mu, mu, 0.0
    s.wall0, s.nwalls, s.tri0, s.ntris = 0, 2, 2, len(tris)
    s.rot_axis[2] = 1.0
    s.rot_omega = -rpm * 2.0 * math.pi / 60.0
    r_in = R - lifter_h - 1.0
    m = 0.05
    sph = lattice_fill(None, (-r_in, -r_in, r_max + m), (r_in, r_in, L - r_max - m),
                       2.0 * r_max + 0.5 * skin, rng)
    sph = sph[np.hypot(sph[:, 0], sph[:, 1]) < r_in - r_max]
    rk = lattice_fill(None, (-r_in, -r_in, rb + m), (r_in, r_in, L - rb - m), 2.0 * rb + 0.05, rng)
    rk = rk[np.hypot(rk[:, 0], rk[:, 1]) < r_in - rb]
    sph, sph_r, rocks = _mixed_placement(rng, sph, rk, n_spheres, n_rocks, r_min, r_max, rbs, 1)
    pos, rad, shape_of, quat = mixed_charge_state(sph, sph_r, rocks, shapes, rng)
    return [s], walls, pos, rad, shapes, shape_of, quat
