"""Generators of the synthetic workloads that the GPU tests and the bench
build on: counts, geometry and the parameters the reference's parser derives
from the projects they write.  No GPU needed."""
import math
import tempfile

import numpy as np

from blaze import synth


def test_drum_mesh_is_the_c3_mesh():
    S, W, p, r = synth.drum_mesh_ensemble(n=2000)
    s = S[0]
    assert s.ntris == 16384 and s.nwalls == 2 and s.tri0 == 2
    assert abs(s.rot_omega + math.pi) < 1e-6          # 30 rpm, clockwise about +z
    tri = np.array([[W[k].p[q] for q in range(9)] for k in range(s.tri0, s.tri0 + s.ntris)])
    v = tri.reshape(-1, 3, 3)
    rr = np.hypot(v[..., 0], v[..., 1])
    # barrel vertices on the drum, lifter vertices inside it, all within its length
    assert rr.max() <= 50.0 + 1e-4 and v[..., 2].min() >= -1e-6 and v[..., 2].max() <= 30.0 + 1e-6
    # every sphere inside the lifter ring, clear of the end plates
    assert np.hypot(p[:, 0], p[:, 1]).max() + r.max() < 50.0 - 4.0
    assert p[:, 2].min() - r.max() > 0.0 and p[:, 2].max() + r.max() < 30.0
    # no two spheres start in contact
    from scipy.spatial import cKDTree
    pairs = np.array(sorted(cKDTree(p.astype(np.float64)).query_pairs(1.3)), dtype=np.int64)
    assert len(pairs) > 0
    d = np.linalg.norm(p[pairs[:, 0]] - p[pairs[:, 1]], axis=1)
    assert np.all(d >= r[pairs[:, 0]] + r[pairs[:, 1]])


def test_box_system_project_matches_the_system():
    S, W, p, r = synth.box_ensemble([500], seed=7)
    edges = np.linspace(0.1, 0.2, 7)
    rb = (0.5 * (edges[:-1] + edges[1:])).astype(np.float32)[np.clip(np.digitize(r, edges) - 1, 0, 5)]
    L, H = -W[1].p[3], -W[5].p[3]
    with tempfile.TemporaryDirectory() as d:
        P, types = synth.box_system_project(d, "Sys", S[0], L, H, rb, 2500.0)
    assert not P.stream_failed and P.num_particles == 500
    si = P.sim_info
    # one cell count on every axis (the reference's hash overruns when nx < nz)
    assert si.num_NNCells.x == si.num_NNCells.y == si.num_NNCells.z
    # the particle objects carry the system's radii and constants
    radii = np.array([P.pobj[t].radius for t in range(P.n_p)], np.float32)
    np.testing.assert_array_equal(radii[types], rb)
    for t in range(P.n_p):
        assert P.pobj[t].PP[t].Kn == np.float32(S[0].kn)
        assert P.pobj[t].PP[t].Fric_kinetic == np.float32(S[0].mu)
        # the parser's mass against (4/3 pi density) r^3 in double
        m = 4.0 / 3.0 * math.pi * float(P.pobj[t].radius) ** 3 * 2500e-6
        assert abs(P.pobj[t].mass - m) <= 2e-7 * m
    # the six faces are the system's six planes
    normals = sorted(tuple(round(v, 6) for v in (f.normal.x, f.normal.y, f.normal.z))
                     for f in list(P.wobj[0].surfaces)[:6])
    planes = sorted(tuple(round(W[k].p[q], 6) for q in range(3)) for k in range(6))
    assert [tuple(abs(x) for x in n) for n in normals] == [tuple(abs(x) for x in n) for n in planes]
