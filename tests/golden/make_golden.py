"""Generate the golden fixtures under tests/golden/ from the reference's own
project files and the reference's own kernels (oracle A: the reference's
DEM kernels compiled as host C++, oracle/_ref/libblaze_refhost.so).

Run in a container that has the reference tree (its path is the first
argument, default $BLAZE_REFERENCE, else a directory "reference" beside the
repository) after `make -C oracle ref`:

    python tests/golden/make_golden.py [/path/to/reference] [fixture ...]

Each fixture is an .npz with
  wobj, pobj, dobj, sim_info   raw bytes of the boundary structs as this
                               project's parser builds them (checked field by
                               field against the reference's parser)
  n_w, n_p, n_d, cyl_rot       counts and the drum-rotation flag
  init_*                       the initial state read from the fixture file
  s{K}_*                       oracle A after K steps: pos, vel, avel, type,
                               pid, the force arrays of step K before
                               integration, and the contact list of step K
Polyhedron fixtures add init_quat / s{K}_quat (w, x, y, z); their positions
are the reference's outputs (pos - COM), their inputs centres of mass.
"""
import ctypes as C
import os
import re
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "softx-d-15-00085_b200"))

from bindings import RefHost  # noqa: E402
import canon  # noqa: E402
from blaze.project import Project  # noqa: E402

CHECKPOINTS = (1, 2, 10, 100)

# (fixture name, project, world, drum rotation on)
FIXTURES = [
    ("silo_sph90", "2.Silo", "SPH_90", False),
    ("mill_sph30", "3.BallMill", "Mill_SPH30", True),
]


def make(ref_root, name, project, world, cyl_rot):
    projects = os.path.join(ref_root, "Projects")
    P = Project.load(projects, project, world)
    R = RefHost()
    rp, w, p, d = R.parse(projects, project, world)
    # the project-input mirror must agree with the reference's parser
    assert [canon.wobj(w[i]) for i in range(rp.n_w)] == [canon.wobj(P.wobj[i]) for i in range(P.n_w)]
    assert [canon.pobj_sphere(p[i], rp.n_p) for i in range(rp.n_p)] == \
        [canon.pobj_sphere(P.pobj[i], P.n_p) for i in range(P.n_p)]
    assert [canon.dobj(d[i]) for i in range(rp.n_d)] == [canon.dobj(P.dobj[i]) for i in range(P.n_d)]
    st = P.read_state()
    R.init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=4, capture=True)
    R.set_cylinder_rotation(cyl_rot)
    R.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    out = dict(
        wobj=np.frombuffer(bytes(P.wobj), np.uint8), pobj=np.frombuffer(bytes(P.pobj), np.uint8),
        dobj=np.frombuffer(bytes(P.dobj), np.uint8),
        sim_info=np.frombuffer(bytes(P.sim_info), np.uint8),
        n_w=P.n_w, n_p=P.n_p, n_d=P.n_d, cyl_rot=int(cyl_rot),
        init_pos=st["pos"], init_vel=st["vel"], init_avel=st["avel"], init_type=st["type"],
        init_pid=st["pid"], source="%s/World/%s.World" % (project, world))
    done = 0
    for k in CHECKPOINTS:
        rc = R.step(k - done)
        assert rc == 0, rc
        done = k
        s = R.state()
        f = R.forces()
        nn, lst = R.nlist()
        for key in ("pos", "vel", "avel", "type", "pid"):
            out["s%d_%s" % (k, key)] = s[key]
        for key, v in f.items():
            out["s%d_%s" % (k, key)] = v
        out["s%d_nn" % k] = nn
        out["s%d_list" % k] = lst[:, :max(1, int(nn.max()))]
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def random_quaternions(rng, n):
    """Uniformly distributed unit quaternions (w, x, y, z), w >= 0."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1.0
    return q.astype(np.float32)


# (fixture name, project, world, particles, lattice spacing cm, seed)
POLY_FIXTURES = [
    ("box_poly", "1.Particles_Box", "Poly_128cm", 1440, 0.93, 7),
]
POLY_CHECKPOINTS = (1, 2, 10, 50)


def make_poly(ref_root, name, project, world, n, spacing, seed):
    """Dodecahedra of the project's own object file on a jittered lattice
    just above the floor of its container, random orientations and
    velocities, so the first steps hold vertex-face, edge-face, face-face and
    edge-edge contacts between particles and with the floor.  The particle
    count replaces the world file's (8,192, lattice-filled and falling for
    thousands of steps before the first contact)."""
    projects = os.path.join(ref_root, "Projects")
    P = Project.load(projects, project, world)
    rp, w, p, d = RefHost.parse_isolated(projects, project, world)
    assert canon.pobj_poly(p[0], 1) == canon.pobj_poly(
        _unscaled(P.pobj[0], p[0]), 1), "project mirror differs from the reference parser"
    P.sim_info.Num_Particles = n
    P.per_object[0] = n
    rng = np.random.default_rng(seed)
    nx = nz = 12
    ny = (n + nx * nz - 1) // (nx * nz)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                 axis=-1).reshape(-1, 3)[:n]
    r_b = float(P.pobj[0].radius)
    base = np.array([60.0, 0.94 * r_b, 60.0])
    pos = (base + g * spacing + rng.uniform(-0.02, 0.02, size=(n, 3))).astype(np.float32)
    quat = random_quaternions(rng, n)
    vel = rng.normal(scale=10.0, size=(n, 3)).astype(np.float32)
    avel = rng.normal(scale=20.0, size=(n, 3)).astype(np.float32)
    ptype = np.zeros(n, np.uint32)
    pid = np.arange(n, dtype=np.int32)
    R = RefHost()
    R.init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=8, capture=True)
    R.set_state(pos, vel, avel, ptype, pid, quat=quat)
    out = dict(
        wobj=np.frombuffer(bytes(P.wobj), np.uint8), pobj=np.frombuffer(bytes(P.pobj), np.uint8),
        dobj=np.frombuffer(bytes(P.dobj), np.uint8),
        sim_info=np.frombuffer(bytes(P.sim_info), np.uint8),
        n_w=P.n_w, n_p=P.n_p, n_d=P.n_d, cyl_rot=0,
        init_pos=pos, init_vel=vel, init_avel=avel, init_quat=quat, init_type=ptype,
        init_pid=pid, source="%s/World/%s.World, %d particles, seed %d" % (project, world, n, seed))
    done = 0
    for k in POLY_CHECKPOINTS:
        rc = R.step(k - done)
        assert rc == 0, rc
        done = k
        s = R.state()
        f = R.forces()
        nn, lst = R.nlist()
        for key in ("pos", "quat", "vel", "avel", "type", "pid"):
            out["s%d_%s" % (k, key)] = s[key]
        for key, v in f.items():
            out["s%d_%s" % (k, key)] = v
        out["s%d_nn" % k] = nn
        out["s%d_list" % k] = lst[:, :max(1, int(nn.max()))]
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def poly_drum_project(ref_root, dst, n, lifters=False):
    """A polyhedron project assembled from the reference's own pieces: the
    90 cm mill drum with both end plates (3.BallMill Drum90cm.WOBJ) filled
    with the dodecahedron of 1.Particles_Box (Poly_1cm.POBJ), the world file
    of Mill_SPH30 with particle type 1, n particles, no lifters and 1 cm
    cells.
    Returns (projects root, project, world)."""
    src = os.path.join(ref_root, "Projects")
    proj = os.path.join(dst, "Projects", "MillPoly")
    for sub in ("World", "SurfaceObjects", "ParticleObjects", "LifterObjects"):
        os.makedirs(os.path.join(proj, sub), exist_ok=True)
    shutil.copy(os.path.join(src, "3.BallMill", "SurfaceObjects", "Drum90cm.WOBJ"),
                os.path.join(proj, "SurfaceObjects"))
    shutil.copy(os.path.join(src, "1.Particles_Box", "ParticleObjects", "Poly_1cm.POBJ"),
                os.path.join(proj, "ParticleObjects"))
    shutil.copy(os.path.join(src, "3.BallMill", "LifterObjects", "Square_Lifter16.DOBJ"),
                os.path.join(proj, "LifterObjects"))
    text = open(os.path.join(src, "3.BallMill", "World", "Mill_SPH30.World")).read()
    reps = [("Particle_Type(0=sphere,1=poly,2=mixed): 0", "Particle_Type(0=sphere,1=poly,2=mixed): 1"),
            ("1 Ball_5cm  242", "1 Poly_1cm  %d" % n),
            ("Num_Particles:    242", "Num_Particles:    %d" % n),
            ("Cell_Size:     5.0   5.0    5.0", "Cell_Size:     1.0   1.0    1.0")]
    for a, b in reps:
        assert a in text, a
        text = text.replace(a, b)
    if not lifters:
        text, k = re.subn(r"Number: 1 Repeat: 8\s+1 Square_Lifter16", "Number: 0 Repeat: 0", text)
        assert k == 1
    open(os.path.join(proj, "World", "Mill_POLY.World"), "w").write(text)
    return os.path.join(dst, "Projects"), "MillPoly", "Mill_POLY"


def make_poly_drum(ref_root, name, n, seed, lifters=False):
    """Dodecahedra in the bottom of the rotating mill drum: drum wall
    (moving-surface law), both end plates, particle contacts, and with
    `lifters` the reference's eight Square_Lifter16 volume objects."""
    tmp = tempfile.mkdtemp(prefix="blaze_polydrum_")
    try:
        projects, project, world = poly_drum_project(ref_root, tmp, n, lifters)
        P = Project.load(projects, project, world)
        rp, w, p, d = RefHost.parse_isolated(projects, project, world)
        assert canon.pobj_poly(p[0], 1) == canon.pobj_poly(_unscaled(P.pobj[0], p[0]), 1)
        assert canon.wobj(w[0]) == canon.wobj(P.wobj[0])
        assert rp.n_d == P.n_d
        for i in range(P.n_d):
            assert canon.dobj(d[i]) == canon.dobj(P.dobj[i])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    rng = np.random.default_rng(seed)
    cyl = P.wobj[0].cyl_geo
    R = float(cyl.radius)
    cx, cy = float(cyl.center_bot_cap.x), float(cyl.center_bot_cap.y)
    H = float(cyl.height)
    r_b = float(P.pobj[0].radius)
    sp = 0.93
    cand = []
    # rings about the drum axis from the wall inwards, in the lowest 40
    # degrees of arc, the outer ring close enough for vertices to reach the
    # wall; z layers between the end plates
    for ring in range(12):
        rad = R - 0.91 * r_b - ring * sp
        dth = sp / rad
        for th in np.arange(-0.35, 0.35, dth):
            for z in np.arange(0.94 * r_b, H - 0.94 * r_b, sp):
                cand.append((cx + rad * np.sin(th), cy - rad * np.cos(th), z))
    cand = np.array(cand)
    cand = (cand + rng.uniform(-0.02, 0.02, size=cand.shape)).astype(np.float32)
    qc = random_quaternions(rng, len(cand))
    if P.n_d:
        keep = lifter_safe(P, cand, qc)
        cand, qc = cand[keep], qc[keep]
    assert len(cand) >= n, len(cand)
    pos, quat = cand[:n], qc[:n]
    vel = rng.normal(scale=10.0, size=(n, 3)).astype(np.float32)
    avel = rng.normal(scale=20.0, size=(n, 3)).astype(np.float32)
    ptype = np.zeros(n, np.uint32)
    pid = np.arange(n, dtype=np.int32)
    Rh = RefHost()
    Rh.init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=8, capture=True)
    Rh.set_cylinder_rotation(True)
    Rh.set_state(pos, vel, avel, ptype, pid, quat=quat)
    out = dict(
        wobj=np.frombuffer(bytes(P.wobj), np.uint8), pobj=np.frombuffer(bytes(P.pobj), np.uint8),
        dobj=np.frombuffer(bytes(P.dobj), np.uint8),
        sim_info=np.frombuffer(bytes(P.sim_info), np.uint8),
        n_w=P.n_w, n_p=P.n_p, n_d=P.n_d, cyl_rot=1,
        init_pos=pos, init_vel=vel, init_avel=avel, init_quat=quat, init_type=ptype,
        init_pid=pid, source="Drum90cm.WOBJ + Poly_1cm.POBJ, %d particles, seed %d" % (n, seed))
    done = 0
    for k in POLY_CHECKPOINTS:
        rc = Rh.step(k - done)
        assert rc == 0, rc
        done = k
        st = Rh.state()
        f = Rh.forces()
        nn, lst = Rh.nlist()
        for key in ("pos", "quat", "vel", "avel", "type", "pid"):
            out["s%d_%s" % (k, key)] = st[key]
        for key, v in f.items():
            out["s%d_%s" % (k, key)] = v
        out["s%d_nn" % k] = nn
        out["s%d_list" % k] = lst[:, :max(1, int(nn.max()))]
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def rotate(q, v):
    """Rotate body-frame points v (k, 3) by unit quaternion q (w, x, y, z)."""
    w, x, y, z = (float(c) for c in q)
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    return v @ R.T


def lifter_safe(P, pos, quat, margin=0.005):
    """Sites whose particle either meets no volume object's bounding
    cylinder, or is cut off from it by a face plane (all vertices at least
    `margin` in front), or has one or two vertices behind all of its faces
    with a `margin` either way: the contacts the reference resolves with its
    vertex-face and edge-face tests.  Deeper contacts can overflow the
    reference's 8-entry vertex arrays, and edge-only ones can leave its
    normal unset, so the fixture starts without them."""
    o = P.pobj[0]
    lv = np.array([[o.Local_Vertex[k].x, o.Local_Vertex[k].y, o.Local_Vertex[k].z]
                   for k in range(o.num_vertex)])
    r_b = float(o.radius)
    keep = np.ones(len(pos), bool)
    for i in range(len(pos)):
        p = pos[i].astype(np.float64)
        for d in range(P.n_d):
            D = P.dobj[d]
            com = np.array([D.COM.x, D.COM.y, D.COM.z])
            ax = np.array([D.Axis.x, D.Axis.y, D.Axis.z])
            if np.linalg.norm((p - com) * ax) >= float(D.boundR) + r_b + margin:
                continue
            v = rotate(quat[i], lv) + p
            dist = []
            for f in range(D.num_faces):
                S = D.faces[f]
                n = np.array([S.normal.x, S.normal.y, S.normal.z])
                c = np.array([S.centroid.x, S.centroid.y, S.centroid.z])
                dist.append((v - c) @ n)
            dist = np.array(dist)
            if np.any(np.all(dist >= margin, axis=1)):
                continue  # one lifter face has every vertex well in front
            inside_hi = int(np.all(dist <= margin, axis=0).sum())
            inside_lo = int(np.all(dist <= -margin, axis=0).sum())
            if not (inside_lo == inside_hi and 1 <= inside_hi <= 2):
                keep[i] = False
                break
    return keep


def _unscaled(mine, ref):
    """The mirror's object with the parser's inertia tensor (the run setup
    scales it afterwards; the scaling has its own test)."""
    c = type(mine).from_buffer_copy(bytes(mine))
    for g in range(9):
        c.InertiaT[g] = ref.InertiaT[g]
    return c


def make_grid(ref_root, name, project, world, projects_dir=None):
    """A world that reads no state file: the boundary structs, its
    InitConfig and the particle count per object (the initial lattice is
    laid out by Device_Set_SimulationData, DeviceInterface.cu:1772-1786)."""
    P = Project.load(projects_dir or os.path.join(ref_root, "Projects"), project, world)
    assert not P.init.use_file
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        wobj=np.frombuffer(bytes(P.wobj), np.uint8), pobj=np.frombuffer(bytes(P.pobj), np.uint8),
        dobj=np.frombuffer(bytes(P.dobj), np.uint8),
        sim_info=np.frombuffer(bytes(P.sim_info), np.uint8),
        init=np.frombuffer(bytes(P.init), np.uint8), n_w=P.n_w, n_p=P.n_p, n_d=P.n_d,
        per_object=np.array([P.per_object[i] for i in range(P.n_p)], np.int32),
        source="%s/World/%s.World" % (project, world))


def make_mill_fill(ref_root, name):
    """The ball mill filled by waves: Mill_SPH30 with its initial setup
    switched to the fill the reference's Mill_SPH30_Fill world asks for
    (Read_FromFile 0, SetpUp 2, launch_Vel 10 -200 10; that world file
    itself lacks its Delta_t line, which its parser then misreads)."""
    with tempfile.TemporaryDirectory() as tmp:
        proj = os.path.join(tmp, "3.BallMill")
        shutil.copytree(os.path.join(ref_root, "Projects", "3.BallMill"), proj)
        wf = os.path.join(proj, "World", "Mill_SPH30.World")
        text = open(wf).read()
        text, k = re.subn(r"Read_FromFile:\s+1\s+File_Name:\s+\S+",
                          "Read_FromFile:  0\nSetpUp(0=grid,2=fill): 2\nlaunch_Vel: 10.0 -200.0 10.0",
                          text)
        assert k == 1
        with open(os.path.join(proj, "World", "Mill_Fill.World"), "w") as fh:
            fh.write(text)
        make_grid(tmp, name, "3.BallMill", "Mill_Fill", projects_dir=tmp)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "BLAZE_REFERENCE", os.path.join(os.path.dirname(REPO), "reference"))
    which = sys.argv[2:] or None
    if which is None or "box_grid" in which:
        make_grid(ref_root, "box_grid", "1.Particles_Box", "Spheres_128cm")
    if which is None or "mill_fill" in which:
        make_mill_fill(ref_root, "mill_fill")
    for name, project, world, rot in FIXTURES:
        if which is None or name in which:
            make(ref_root, name, project, world, rot)
    for name, project, world, n, spacing, seed in POLY_FIXTURES:
        if which is None or name in which:
            make_poly(ref_root, name, project, world, n, spacing, seed)
    if which is None or "drum_poly" in which:
        make_poly_drum(ref_root, "drum_poly", 1200, 11)
    if which is None or "lifter_poly" in which:
        make_poly_drum(ref_root, "lifter_poly", 1200, 13, lifters=True)


if __name__ == "__main__":
    main()
